// Learned vertical-mixing closure: BF16 tensor-core inference on sm_100a
// (tcgen05.mma, accumulators in tensor memory, FP32 accumulation).  No
// counterpart in the reference; the network stands in for d3_end
// (src/fv_mixing.F90:73-347).
//
// One persistent CTA per SM (128 threads, 4 warps) walks 128-column tiles.
// Per tile: the normalised inputs (FP32) are converted to BF16 into shared
// memory; four layers of tcgen05.mma (M = 128 columns, N = output neurons,
// K = 16 per instruction) accumulate in TMEM (256 of the SM's 512 columns);
// after each layer the four warps read their 32 TMEM lanes (tcgen05.ld),
// add the bias, apply SiLU and write the BF16 activations back to shared
// memory as the next layer's A operand; the last layer's FP32 outputs go to
// global memory.  W1 and W4 stay in shared memory for the kernel's life;
// W2 and W3 (128 KB each) stream through one 64 KB buffer in halves of 128
// output neurons (they stay in L2, every CTA reads the same 256 KB).
//
// Operands use the no-swizzle K-major canonical layout: 8-row x 16-byte
// core matrices, an operand of R rows stored as K/8 slabs of R x 16 bytes
// ("chunk-major"): element (r, k) at byte (k/8)*R*16 + r*16 + (k%8)*2.  The
// descriptor of the k-th 16-wide slice starts at slab 2k, with LBO = R*16
// (the next 8-wide chunk) and SBO = 128 (the next 8 rows).  The host lays
// the BF16 weights out the same way, so their copies are contiguous.
//
// Every wait on the MMA-completion barrier is bounded; a CTA whose MMAs do
// not complete in about a second sets the error word, frees its tensor
// memory and returns.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "closure.h"
#include "mlp.h"

namespace fesomc {
namespace {

constexpr int kTM = 128;                 // columns per tile (MMA M)
constexpr int kThreads = 128;
constexpr int kSlab = kTM * 16;          // bytes of one 8-wide K chunk of a 128-row operand
constexpr uint32_t kTmemCols = 256;

struct TcParams {
    int IN, OUT, K1p, N4p;
    long long ncol;
    const float *X;                      // ncol x IN, normalised FP32
    float *Y;                            // ncol x OUT, FP32
    const uint4 *W1, *W2, *W3, *W4;      // BF16, chunk-major
    const float *b1, *b2, *b3, *b4;
    unsigned int *err;
    // shared-memory offsets (bytes)
    int oX, oH, oW1, oW4, oWB, oB, oBar;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor, no swizzle, K-major (version 1)
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: BF16 A and B (K-major), FP32 accumulator, M = 128
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTM >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accum));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// bounded wait for the barrier phase; false on timeout (about a second)
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t phase) {
    for (uint32_t it = 0; it < (1u << 25); ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done) return true;
        __nanosleep(32);
    }
    return false;
}

// 32 consecutive TMEM columns of this warp's 32 lanes
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    wait_ld();
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float silu_dev(float z) { return z / (1.0f + expf(-z)); }

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&h);
}

// copy n16 16-byte words from global to shared
__device__ __forceinline__ void copy_words(uint4 *dst, const uint4 *src, int n16) {
    for (int i = threadIdx.x; i < n16; i += kThreads) dst[i] = __ldg(src + i);
}

// bias + SiLU of the 256 accumulator columns of this thread's row, to the
// BF16 activation operand (row r, chunk-major, 128 rows)
__device__ __forceinline__ void epi_hidden(uint32_t tbase, unsigned char *H, const float *bias) {
    const int w = threadIdx.x >> 5, r = threadIdx.x;
    for (int c0 = 0; c0 < 256; c0 += 32) {
        float v[32];
        tmem_ld32(tbase + ((uint32_t)(32 * w) << 16) + (uint32_t)c0, v);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint4 o;
            o.x = pack_bf16(silu_dev(v[8 * q + 0] + bias[c0 + 8 * q + 0]), silu_dev(v[8 * q + 1] + bias[c0 + 8 * q + 1]));
            o.y = pack_bf16(silu_dev(v[8 * q + 2] + bias[c0 + 8 * q + 2]), silu_dev(v[8 * q + 3] + bias[c0 + 8 * q + 3]));
            o.z = pack_bf16(silu_dev(v[8 * q + 4] + bias[c0 + 8 * q + 4]), silu_dev(v[8 * q + 5] + bias[c0 + 8 * q + 5]));
            o.w = pack_bf16(silu_dev(v[8 * q + 6] + bias[c0 + 8 * q + 6]), silu_dev(v[8 * q + 7] + bias[c0 + 8 * q + 7]));
            *reinterpret_cast<uint4 *>(H + (size_t)(c0 / 8 + q) * kSlab + (size_t)r * 16) = o;
        }
    }
}

__global__ void __launch_bounds__(kThreads, 1) k_mlp_tc(TcParams p) {
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char *sX = sm + p.oX, *sH = sm + p.oH, *sW1 = sm + p.oW1, *sW4 = sm + p.oW4, *sWB = sm + p.oWB;
    float *sb = reinterpret_cast<float *>(sm + p.oB);          // b1 b2 b3 (256 each), b4 (N4p)
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + p.oBar);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + p.oBar + 8);
    int *sfail = reinterpret_cast<int *>(sm + p.oBar + 12);
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t bar_a = smem_u32(bar);

    // resident weights and biases
    copy_words(reinterpret_cast<uint4 *>(sW1), p.W1, 256 * p.K1p * 2 / 16);
    copy_words(reinterpret_cast<uint4 *>(sW4), p.W4, p.N4p * 256 * 2 / 16);
    for (int i = tid; i < 256; i += kThreads) {
        sb[i] = p.b1[i];
        sb[256 + i] = p.b2[i];
        sb[512 + i] = p.b3[i];
    }
    for (int i = tid; i < p.N4p; i += kThreads) sb[768 + i] = i < p.OUT ? p.b4[i] : 0.0f;
    if (tid == 0) {
        *sfail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_proxy();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tbase = *tslot;
    uint32_t phase = 0;
    const long long ntiles = (p.ncol + kTM - 1) / kTM;
    const uint32_t id256 = idesc_bf16(256), id128 = idesc_bf16(128), idN4 = idesc_bf16(p.N4p);
    const uint32_t aX = smem_u32(sX), aH = smem_u32(sH), aW1 = smem_u32(sW1), aW4 = smem_u32(sW4), aWB = smem_u32(sWB);
    bool ok = true;

    // wait for the MMAs committed so far; all threads agree on the outcome
    auto wait_mma = [&]() {
        const bool done = bar_wait(bar_a, phase);
        phase ^= 1u;
        if (!done) atomicOr(sfail, 1);
        __syncthreads();
        ok = ok && (*sfail == 0);
        fence_after();
    };

    for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const long long row0 = tile * kTM;
        // inputs of this tile to BF16 (zero rows beyond ncol, zero K padding)
        {
            const long long row = row0 + tid;
            const bool valid = row < p.ncol;
            const float *x = p.X + (valid ? row : 0) * p.IN;
            for (int kc = 0; kc < p.K1p / 8; ++kc) {
                float v[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int k = kc * 8 + j;
                    v[j] = (valid && k < p.IN) ? x[k] : 0.0f;
                }
                uint4 o;
                o.x = pack_bf16(v[0], v[1]);
                o.y = pack_bf16(v[2], v[3]);
                o.z = pack_bf16(v[4], v[5]);
                o.w = pack_bf16(v[6], v[7]);
                *reinterpret_cast<uint4 *>(sX + (size_t)kc * kSlab + (size_t)tid * 16) = o;
            }
        }
        fence_proxy();
        fence_before();
        __syncthreads();
        // layer 1: [128 x K1p] x [K1p x 256]
        if (tid == 0) {
            fence_after();
            for (int s = 0; s < p.K1p / 16; ++s)
                mma_bf16(tbase, sdesc(aX + 2 * s * kSlab, kSlab, 128), sdesc(aW1 + 2 * s * 256 * 16, 256 * 16, 128),
                         id256, s > 0);
            mma_commit(bar_a);
        }
        wait_mma();
        if (!ok) break;
        epi_hidden(tbase, sH, sb);
        // layers 2 and 3: [128 x 256] x [256 x 256], W in two halves of 128 neurons
        for (int l = 0; l < 2 && ok; ++l) {
            const uint4 *W = l == 0 ? p.W2 : p.W3;
            for (int half = 0; half < 2; ++half) {
                copy_words(reinterpret_cast<uint4 *>(sWB), W + (size_t)half * (128 * 256 * 2 / 16), 128 * 256 * 2 / 16);
                fence_proxy();
                wait_ld();
                fence_before();
                __syncthreads();
                if (tid == 0) {
                    fence_after();
                    for (int s = 0; s < 16; ++s)
                        mma_bf16(tbase + (uint32_t)(128 * half), sdesc(aH + 2 * s * kSlab, kSlab, 128),
                                 sdesc(aWB + 2 * s * 128 * 16, 128 * 16, 128), id128, s > 0);
                    mma_commit(bar_a);
                }
                wait_mma();
                if (!ok) break;
            }
            if (!ok) break;
            epi_hidden(tbase, sH, sb + 256 * (l + 1));
        }
        if (!ok) break;
        fence_proxy();
        fence_before();
        __syncthreads();
        // layer 4: [128 x 256] x [256 x N4p]
        if (tid == 0) {
            fence_after();
            for (int s = 0; s < 16; ++s)
                mma_bf16(tbase, sdesc(aH + 2 * s * kSlab, kSlab, 128), sdesc(aW4 + 2 * s * p.N4p * 16, p.N4p * 16, 128),
                         idN4, s > 0);
            mma_commit(bar_a);
        }
        wait_mma();
        if (!ok) break;
        {
            const long long row = row0 + tid;
            for (int c0 = 0; c0 < p.N4p; c0 += 32) {
                float v[32];
                tmem_ld32(tbase + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
                if (row < p.ncol)
                    for (int j = 0; j < 32 && c0 + j < p.OUT; ++j) p.Y[row * p.OUT + c0 + j] = v[j] + sb[768 + c0 + j];
            }
        }
        fence_before();
        __syncthreads();
    }
    if (!ok) {
        if (tid == 0) atomicOr(p.err, 1u);
        // a commit that timed out may still complete: wait for it once more
        // (bounded) before the tensor memory is given back
        bar_wait(bar_a, phase ^ 1u);
    }
    fence_before();
    __syncthreads();
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(kTmemCols) : "memory");
    }
}

// element (r, k) of an R-row operand in the chunk-major layout, in BF16 units
inline size_t cm_index(int R, int r, int k) { return (size_t)(k / 8) * R * 8 + (size_t)r * 8 + (k % 8); }

uint16_t bf16_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7F800000u) == 0x7F800000u) return (uint16_t)(u >> 16);   // inf / nan
    u += 0x7FFFu + ((u >> 16) & 1u);                                     // round to nearest even
    return (uint16_t)(u >> 16);
}

}  // namespace

static size_t tc_smem(int K1p, int N4p, TcParams *o);

// the kernel's shared-memory plan fits one SM (227 KB): nsigma <= 25
bool lc_tc_supported(const LcNet *n) {
    const int K1p = (n->IN + 15) / 16 * 16, N4p = (n->OUT + 15) / 16 * 16;
    return N4p <= 64 && tc_smem(K1p, N4p, nullptr) <= 232448;
}

static size_t tc_smem(int K1p, int N4p, TcParams *o) {
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t at = off;
        off += (bytes + 1023) / 1024 * 1024;
        return (int)at;
    };
    const int oX = take((size_t)kTM * K1p * 2), oH = take((size_t)kTM * 256 * 2), oW1 = take((size_t)256 * K1p * 2),
              oW4 = take((size_t)N4p * 256 * 2), oWB = take((size_t)128 * 256 * 2),
              oB = take((size_t)(768 + 64) * 4), oBar = take(64);
    if (o) {
        o->oX = oX; o->oH = oH; o->oW1 = oW1; o->oW4 = oW4; o->oWB = oWB; o->oB = oB; o->oBar = oBar;
    }
    return off;
}

// BF16 copies of the weights in the chunk-major operand layout (after every
// parameter change)
int lc_tc_prepare(LcNet *n) {
    if (!lc_tc_supported(n)) return FESOMC_EINVAL_LC;
    const int K1p = (n->IN + 15) / 16 * 16, N4p = (n->OUT + 15) / 16 * 16;
    std::vector<float> p(n->np);
    if (cudaMemcpy(p.data(), n->params, sizeof(float) * n->np, cudaMemcpyDeviceToHost) != cudaSuccess)
        return FESOMC_ECUDA_LC;
    const size_t s1 = (size_t)256 * K1p, s2 = (size_t)256 * 256, s4 = (size_t)N4p * 256;
    std::vector<uint16_t> w(s1 + 2 * s2 + s4, 0);
    // W1: 256 rows (neurons) x K1p
    for (int r = 0; r < 256; ++r)
        for (int k = 0; k < n->IN; ++k) w[cm_index(256, r, k)] = bf16_bits(p[n->off[0] + (size_t)r * n->IN + k]);
    // W2, W3: two halves of 128 neurons, each a 128-row operand
    for (int l = 1; l <= 2; ++l) {
        uint16_t *base = w.data() + s1 + (size_t)(l - 1) * s2;
        for (int r = 0; r < 256; ++r)
            for (int k = 0; k < 256; ++k)
                base[(size_t)(r / 128) * 128 * 256 + cm_index(128, r % 128, k)] =
                    bf16_bits(p[n->off[l] + (size_t)r * 256 + k]);
    }
    uint16_t *b4 = w.data() + s1 + 2 * s2;
    for (int r = 0; r < n->OUT; ++r)
        for (int k = 0; k < 256; ++k) b4[cm_index(N4p, r, k)] = bf16_bits(p[n->off[3] + (size_t)r * 256 + k]);
    if (!n->wtc) {
        void *q = nullptr;
        if (cudaMalloc(&q, w.size() * 2) != cudaSuccess) return FESOMC_ENOMEM_LC;
        n->allocs.push_back(q);
        n->wtc = static_cast<uint16_t *>(q);
        if (cudaMalloc(&q, sizeof(unsigned int)) != cudaSuccess) return FESOMC_ENOMEM_LC;
        n->allocs.push_back(q);
        n->tc_err = static_cast<unsigned int *>(q);
        cudaMemset(n->tc_err, 0, sizeof(unsigned int));
    }
    if (cudaMemcpy(n->wtc, w.data(), w.size() * 2, cudaMemcpyHostToDevice) != cudaSuccess) return FESOMC_ECUDA_LC;
    n->tc_ready = true;
    return 0;
}

// Y (B x OUT) = network(X (B x IN)) with the BF16 tensor-core kernel
int lc_forward_tc(const LcNet *n, const float *X, long long B, float *Y, cudaStream_t s) {
    if (!n->tc_ready) return FESOMC_ESTATE_LC;
    TcParams p{};
    p.IN = n->IN;
    p.OUT = n->OUT;
    p.K1p = (n->IN + 15) / 16 * 16;
    p.N4p = (n->OUT + 15) / 16 * 16;
    p.ncol = B;
    p.X = X;
    p.Y = Y;
    const size_t s1 = (size_t)256 * p.K1p, s2 = (size_t)256 * 256;
    p.W1 = reinterpret_cast<const uint4 *>(n->wtc);
    p.W2 = reinterpret_cast<const uint4 *>(n->wtc + s1);
    p.W3 = reinterpret_cast<const uint4 *>(n->wtc + s1 + s2);
    p.W4 = reinterpret_cast<const uint4 *>(n->wtc + s1 + 2 * s2);
    p.b1 = n->params + n->off[0] + (long long)256 * n->IN;
    p.b2 = n->params + n->off[1] + (long long)256 * 256;
    p.b3 = n->params + n->off[2] + (long long)256 * 256;
    p.b4 = n->params + n->off[3] + (long long)n->OUT * 256;
    p.err = n->tc_err;
    const size_t smem = tc_smem(p.K1p, p.N4p, &p);
    static size_t raised = 0;
    if (smem > raised) {
        if (cudaFuncSetAttribute(k_mlp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return FESOMC_ECUDA_LC;
        raised = smem;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long ntiles = (B + kTM - 1) / kTM;
    const int grid = (int)std::max(1LL, std::min<long long>(ntiles, sms));
    k_mlp_tc<<<grid, kThreads, smem, s>>>(p);
    return cudaGetLastError() == cudaSuccess ? 0 : FESOMC_ECUDA_LC;
}

size_t lc_tc_smem_bytes(const LcNet *n) {
    return tc_smem((n->IN + 15) / 16 * 16, (n->OUT + 15) / 16 * 16, nullptr);
}

}  // namespace fesomc
