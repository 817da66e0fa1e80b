// Learned vertical-mixing closure: BF16 tensor-core inference on sm_100a
// (tcgen05.mma, accumulators in tensor memory, FP32 accumulation).  No
// counterpart in the reference; the network stands in for d3_end
// (src/fv_mixing.F90:73-347).
//
// One persistent CTA per SM walks 128-column tiles, two at a time in
// alternation (tile slots 0 and 1: the CTA's even and odd tiles), with
// specialised warps:
//   warp 0       producer: streams the weights, unit by unit, from global
//                memory (L2-resident: every CTA reads the same ~330 KB) into
//                a ring of kSlots shared-memory slots with bulk copies
//                (cp.async.bulk, completion counted on the slot's mbarrier),
//                in the order the MMAs take them;
//   warp 1       MMA issuer (one lane): layer by layer, alternating between
//                the two tiles, per weight unit K/16 tcgen05.mma (M = 128
//                columns, N = 64 neurons, K = 16) into the tile slot's 256
//                tensor-memory columns, a commit that frees the weight slot,
//                and after the layer's last unit a commit that hands the
//                slot's accumulator over;
//   warps 4-11   epilogue of tile slot 0, warps 12-19 of tile slot 1 (two
//                warps per TMEM lane quarter, 128 of the 256 accumulator
//                columns each, read 64 at a time): the tile's normalised
//                FP32 inputs to BF16 in the slot's shared-memory operand
//                buffer, then per hidden layer bias + SiLU of the
//                accumulator (tcgen05.ld) back into that buffer as the next
//                layer's A operand, and the last layer's FP32 outputs to
//                global memory.
// While one slot's epilogue works, the MMAs run the other slot's layer, so
// the tensor pipe and the epilogue overlap instead of taking turns.  The
// weight units are 64 output neurons x the layer's whole K (W1: 4 units,
// W2, W3: 4 each, W4: 1 of N4p neurons).
//
// Operands use the no-swizzle K-major canonical layout: 8-row x 16-byte
// core matrices, an operand of R rows stored as K/8 slabs of R x 16 bytes
// ("chunk-major"): element (r, k) at byte (k/8)*R*16 + r*16 + (k%8)*2.  The
// descriptor of the k-th 16-wide slice starts at slab 2k, with LBO = R*16
// (the next 8-wide chunk) and SBO = 128 (the next 8 rows).  The host lays
// every weight unit out the same way (R = 64, or N4p for W4), so a unit is
// one contiguous bulk copy.
//
// Every wait on an mbarrier is bounded (about a second); a role that gives
// up sets the CTA's failure flag and the error word, the others see the flag
// and stop, and the CTA waits (bounded) for its own copies and MMAs in
// flight before it frees its tensor memory and returns.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "closure.h"
#include "mlp.h"

namespace fesomc {
namespace {

constexpr int kTM = 128;                  // columns per tile (MMA M)
constexpr int kUnitN = 64;                // output neurons per weight unit (MMA N)
constexpr int kSlots = 2;                 // weight slots in shared memory
constexpr int kSlotBytes = kUnitN * 256 * 2;
constexpr int kGroupWarps = 8;            // epilogue warps per tile slot: 2 per TMEM lane quarter
constexpr int kGroupThreads = 32 * kGroupWarps;
constexpr int kThreads = 128 + 2 * kGroupThreads;
constexpr int kSlab = kTM * 16;           // bytes of one 8-wide K chunk of the 128-row A operand
constexpr int kHBytes = kTM * 256 * 2;    // one tile slot's A operand buffer
constexpr uint32_t kTmemCols = 512;       // two accumulators of 256 columns
constexpr int kMaxUnits = 16;
constexpr uint32_t kSpin = 1u << 25;
// barriers: full[kSlots], empty[kSlots], acc[2], a[2], drain
constexpr int kBars = 2 * kSlots + 5;

struct TcParams {
    int IN, OUT, K1p, N4p;
    long long ncol;
    const float *X;                      // ncol x IN, normalised FP32
    float *Y;                            // ncol x OUT, FP32
    const unsigned char *W;              // BF16 weight units, chunk-major, back to back
    int n_units;
    int unit_off[kMaxUnits];             // byte offset of unit u in W
    int unit_bytes[kMaxUnits];
    int unit_rows[kMaxUnits];            // N of the unit's MMAs
    int unit_k[kMaxUnits];               // K of the unit (K1p or 256)
    int unit_col[kMaxUnits];             // first accumulator column of the unit
    int unit_last[kMaxUnits];            // 1: the last unit of its layer
    int layer_start[5];                  // units of layer l: layer_start[l] .. layer_start[l+1]-1
    const float *b1, *b2, *b3, *b4;
    unsigned int *err;
    // shared-memory offsets (bytes)
    int oH, oW, oB, oBar;
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

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// bulk copy global -> this CTA's shared memory (no multicast), completion
// counted on bar
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// bounded wait for the completion of the barrier phase of the given parity;
// false on timeout, or when fail (if given) is set
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity, const volatile int *fail) {
    for (uint32_t it = 0; it < kSpin; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 255u) == 255u && fail && *fail) return false;
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

// 32 consecutive TMEM columns of this warp's 32 lanes, without the wait:
// two of these are in flight before tmem_wait2
__device__ __forceinline__ void tmem_ld32_async(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}
// the wait for the loads in flight; the registers pass through it, so no
// use of them is scheduled before it
#define R16(a, o) "+r"(a[o + 0]), "+r"(a[o + 1]), "+r"(a[o + 2]), "+r"(a[o + 3]), "+r"(a[o + 4]), "+r"(a[o + 5]), \
    "+r"(a[o + 6]), "+r"(a[o + 7]), "+r"(a[o + 8]), "+r"(a[o + 9]), "+r"(a[o + 10]), "+r"(a[o + 11]),          \
    "+r"(a[o + 12]), "+r"(a[o + 13]), "+r"(a[o + 14]), "+r"(a[o + 15])
__device__ __forceinline__ void tmem_wait2(uint32_t (&a)[32], uint32_t (&b)[32]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;" : R16(a, 0), R16(a, 16), R16(b, 0), R16(b, 16)::"memory");
}
#undef R16

// SiLU as z/2 (1 + tanh(z/2)) with the hardware tanh approximation (one
// special-function operation per activation instead of an exponential and a
// reciprocal: the epilogue is bound by that pipe; the approximation's error,
// about 2^-11 relative, is below the BF16 rounding of the result)
__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float silu_fast(float z) {
    const float h = 0.5f * z;
    return fmaf(h, tanh_approx(h), h);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&h);
}

__device__ __forceinline__ void fail_now(volatile int *fail, unsigned int *err) {
    *fail = 1;
    atomicOr(err, 1u);
}

__global__ void __launch_bounds__(kThreads, 1) k_mlp_tc(const __grid_constant__ TcParams p) {
    extern __shared__ __align__(1024) unsigned char sm[];
    float *sb = reinterpret_cast<float *>(sm + p.oB);          // b1 b2 b3 (256 each), b4 (N4p)
    const uint32_t bar0 = smem_u32(sm + p.oBar);
    auto full_bar = [&](int s) { return bar0 + 8u * (uint32_t)s; };
    auto empty_bar = [&](int s) { return bar0 + 8u * (uint32_t)(kSlots + s); };
    auto acc_bar = [&](int g) { return bar0 + 8u * (uint32_t)(2 * kSlots + g); };
    auto a_bar = [&](int g) { return bar0 + 8u * (uint32_t)(2 * kSlots + 2 + g); };
    const uint32_t drain_bar = bar0 + 8u * (uint32_t)(2 * kSlots + 4);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + p.oBar + 8 * kBars);
    volatile int *sfail = reinterpret_cast<volatile int *>(sm + p.oBar + 8 * kBars + 4);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    for (int i = tid; i < 256; i += kThreads) {
        sb[i] = p.b1[i];
        sb[256 + i] = p.b2[i];
        sb[512 + i] = p.b3[i];
    }
    for (int i = tid; i < p.N4p; i += kThreads) sb[768 + i] = i < p.OUT ? p.b4[i] : 0.0f;
    if (tid == 0) {
        *sfail = 0;
        for (int s = 0; s < kSlots; ++s) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), 1);
        }
        for (int g = 0; g < 2; ++g) {
            mbar_init(acc_bar(g), 1);
            mbar_init(a_bar(g), kGroupWarps);
        }
        mbar_init(drain_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tbase = *tslot;
    const long long ntiles = (p.ncol + kTM - 1) / kTM;
    // this CTA's tiles: k = 0 .. K-1 is tile blockIdx.x + k * gridDim.x, in
    // tile slot k % 2; the k-th pair is tiles 2k (slot 0) and 2k+1 (slot 1)
    const long long K = ntiles > (long long)blockIdx.x ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    if (warp == 0) {
        // ---- producer: the units in the order the MMAs take them ----
        if (lane == 0) {
            long long gu = 0;   // units issued
            bool ok = true;
            for (long long pr = 0; 2 * pr < K && ok; ++pr)
                for (int l = 0; l < 4 && ok; ++l)
                    for (int g = 0; g < 2 && ok; ++g) {
                        if (2 * pr + g >= K) continue;
                        for (int u = p.layer_start[l]; u < p.layer_start[l + 1]; ++u) {
                            const int s = (int)(gu % kSlots);
                            const long long n = gu / kSlots;
                            if (n >= 1 && !bar_wait(empty_bar(s), (uint32_t)((n - 1) & 1), sfail)) {
                                fail_now(sfail, p.err);
                                ok = false;
                                break;
                            }
                            mbar_expect_tx(full_bar(s), (uint32_t)p.unit_bytes[u]);
                            bulk_g2s(smem_u32(sm + p.oW + s * kSlotBytes), p.W + p.unit_off[u],
                                     (uint32_t)p.unit_bytes[u], full_bar(s));
                            ++gu;
                        }
                    }
            // every copy issued lands before the CTA may leave: wait for the
            // phase of each slot's last use (already complete when the MMAs
            // consumed it)
            for (int s = 0; s < kSlots; ++s) {
                const long long uses = gu > s ? (gu - 1 - s) / kSlots + 1 : 0;
                if (uses > 0) bar_wait(full_bar(s), (uint32_t)((uses - 1) & 1), nullptr);
            }
        }
    } else if (warp == 1) {
        // ---- MMA issuer: layer by layer, alternating between the tile slots ----
        if (lane == 0) {
            long long gu = 0, a_uses[2] = {0, 0};
            bool ok = true;
            for (long long pr = 0; 2 * pr < K && ok; ++pr)
                for (int l = 0; l < 4 && ok; ++l)
                    for (int g = 0; g < 2 && ok; ++g) {
                        if (2 * pr + g >= K) continue;
                        // the slot's A operand (inputs or activations) is ready
                        if (!bar_wait(a_bar(g), (uint32_t)(a_uses[g] & 1), sfail)) {
                            fail_now(sfail, p.err);
                            ok = false;
                            break;
                        }
                        ++a_uses[g];
                        const uint32_t aH = smem_u32(sm + p.oH + g * kHBytes);
                        const uint32_t dcol = tbase + (uint32_t)(256 * g);
                        for (int u = p.layer_start[l]; u < p.layer_start[l + 1]; ++u) {
                            const int s = (int)(gu % kSlots);
                            if (!bar_wait(full_bar(s), (uint32_t)((gu / kSlots) & 1), sfail)) {
                                fail_now(sfail, p.err);
                                ok = false;
                                break;
                            }
                            fence_after();
                            const uint32_t aW = smem_u32(sm + p.oW + s * kSlotBytes);
                            const int R = p.unit_rows[u];
                            const uint32_t id = idesc_bf16(R);
                            for (int ks = 0; ks < p.unit_k[u] / 16; ++ks)
                                mma_bf16(dcol + (uint32_t)p.unit_col[u], sdesc(aH + 2 * ks * kSlab, kSlab, 128),
                                         sdesc(aW + 2 * ks * R * 16, (uint32_t)R * 16, 128), id, ks > 0);
                            mma_commit(empty_bar(s));
                            ++gu;
                        }
                        if (ok) mma_commit(acc_bar(g));
                    }
            // every MMA issued completes before the tensor memory is freed
            mma_commit(drain_bar);
            bar_wait(drain_bar, 0, nullptr);
        }
    } else if (warp >= 4) {
        // ---- epilogue of tile slot g ----
        const int g = (warp - 4) / kGroupWarps;
        const int gw = (warp - 4) % kGroupWarps;
        const int q = warp & 3;                     // TMEM lane quarter
        const int part = gw >> 2;                   // half of the accumulator columns
        const int r = 32 * q + lane;                // tile row of this thread
        const int e = tid - 128 - g * kGroupThreads;
        unsigned char *sH = sm + p.oH + g * kHBytes;
        const uint32_t tcol = tbase + (uint32_t)(256 * g) + ((uint32_t)(32 * q) << 16);
        long long acc_uses = 0;
        bool ok = true;
        for (long long k = g; k < K && ok; k += 2) {
            const long long row0 = ((long long)blockIdx.x + k * gridDim.x) * kTM;
            const long long left = p.ncol - row0;
            const int nr = left < kTM ? (int)left : kTM;
            // inputs to BF16, one (8-wide K chunk, row) per item with the row
            // fastest: each item is one 16-byte store (consecutive threads,
            // consecutive rows: no bank conflicts), the K padding zero; rows
            // beyond ncol keep stale values (their outputs are not stored)
            const float *x = p.X + row0 * p.IN;
            for (int i = e; i < (p.K1p / 8) * kTM; i += kGroupThreads) {
                const int kc = i / kTM, rr = i - kc * kTM;
                if (rr >= nr) continue;
                const float *xr = x + (size_t)rr * p.IN + 8 * kc;
                float v[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) v[j] = (8 * kc + j < p.IN) ? __ldg(xr + j) : 0.0f;
                uint4 o;
                o.x = pack_bf16(v[0], v[1]);
                o.y = pack_bf16(v[2], v[3]);
                o.z = pack_bf16(v[4], v[5]);
                o.w = pack_bf16(v[6], v[7]);
                *reinterpret_cast<uint4 *>(sH + (size_t)kc * kSlab + (size_t)rr * 16) = o;
            }
            fence_proxy();
            __syncwarp();
            if (lane == 0) mbar_arrive(a_bar(g));
            for (int l = 0; l < 4; ++l) {
                if (!bar_wait(acc_bar(g), (uint32_t)(acc_uses & 1), sfail)) {
                    fail_now(sfail, p.err);
                    ok = false;
                    break;
                }
                ++acc_uses;
                fence_after();
                if (l < 3) {
                    const float *bias = sb + 256 * l;
                    // this warp's 128 columns, 64 at a time: both loads in flight, one wait
#pragma unroll 1
                    for (int c0 = 128 * part; c0 < 128 * part + 128; c0 += 64) {
                        uint32_t ra[32], rb[32];
                        tmem_ld32_async(tcol + (uint32_t)c0, ra);
                        tmem_ld32_async(tcol + (uint32_t)(c0 + 32), rb);
                        tmem_wait2(ra, rb);
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const uint32_t *rv = h == 0 ? ra : rb;
                            const int cb = c0 + 32 * h;
#pragma unroll
                            for (int j = 0; j < 4; ++j) {
                                float v[8];
#pragma unroll
                                for (int t = 0; t < 8; ++t)
                                    v[t] = silu_fast(__uint_as_float(rv[8 * j + t]) + bias[cb + 8 * j + t]);
                                uint4 o;
                                o.x = pack_bf16(v[0], v[1]);
                                o.y = pack_bf16(v[2], v[3]);
                                o.z = pack_bf16(v[4], v[5]);
                                o.w = pack_bf16(v[6], v[7]);
                                *reinterpret_cast<uint4 *>(sH + (size_t)(cb / 8 + j) * kSlab + (size_t)r * 16) = o;
                            }
                        }
                    }
                    fence_before();
                    fence_proxy();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(a_bar(g));
                } else {
                    const long long row = row0 + r;
                    for (int c0 = 32 * part; c0 < p.N4p; c0 += 64) {
                        float v[32];
                        tmem_ld32(tcol + (uint32_t)c0, v);
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            if (row < p.ncol && c0 + j < p.OUT) p.Y[row * p.OUT + c0 + j] = v[j] + sb[768 + c0 + j];
                    }
                    fence_before();
                }
            }
        }
    }
    __syncwarp();
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

// the weight units of the network, in the order the kernel consumes them
struct UnitPlan {
    int n = 0;
    int off[kMaxUnits], bytes[kMaxUnits], rows[kMaxUnits], k[kMaxUnits], col[kMaxUnits], last[kMaxUnits];
    int layer[kMaxUnits], first_neuron[kMaxUnits];
    size_t total = 0;
};

UnitPlan unit_plan(int K1p, int N4p) {
    UnitPlan u;
    auto add = [&](int layer, int rows, int k, int col, int first, bool last) {
        const int i = u.n++;
        u.off[i] = (int)u.total;
        u.bytes[i] = rows * k * 2;
        u.rows[i] = rows;
        u.k[i] = k;
        u.col[i] = col;
        u.last[i] = last ? 1 : 0;
        u.layer[i] = layer;
        u.first_neuron[i] = first;
        u.total += (size_t)u.bytes[i];
    };
    for (int j = 0; j < 4; ++j) add(0, kUnitN, K1p, kUnitN * j, kUnitN * j, j == 3);
    for (int l = 1; l <= 2; ++l)
        for (int j = 0; j < 4; ++j) add(l, kUnitN, 256, kUnitN * j, kUnitN * j, j == 3);
    add(3, N4p, 256, 0, 0, true);
    return u;
}

size_t tc_smem(int IN, TcParams *o) {
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t at = off;
        off += (bytes + 1023) / 1024 * 1024;
        return (int)at;
    };
    (void)IN;
    const int oH = take((size_t)2 * kHBytes), oW = take((size_t)kSlots * kSlotBytes),
              oB = take((size_t)(768 + 64) * 4), oBar = take(8 * kBars + 8);
    if (o) {
        o->oH = oH; o->oW = oW; o->oB = oB; o->oBar = oBar;
    }
    return off;
}

int k1p_of(const LcNet *n) { return (n->IN + 15) / 16 * 16; }
int n4p_of(const LcNet *n) { return (n->OUT + 15) / 16 * 16; }

}  // namespace

// the kernel's plan: the first layer's K fits a weight slot and the outputs
// one unit (nsigma <= 32 at 3*nsigma + 3 inputs and 2*nsigma outputs), the
// shared memory fits one SM
bool lc_tc_supported(const LcNet *n) {
    return k1p_of(n) <= 256 && n4p_of(n) <= kUnitN && tc_smem(n->IN, nullptr) <= 232448;
}

// BF16 copies of the weights as the kernel's units (after every parameter
// change)
int lc_tc_prepare(LcNet *n) {
    if (!lc_tc_supported(n)) return FESOMC_EINVAL_LC;
    const int K1p = k1p_of(n), N4p = n4p_of(n);
    std::vector<float> p(n->np);
    if (cudaMemcpy(p.data(), n->params, sizeof(float) * n->np, cudaMemcpyDeviceToHost) != cudaSuccess)
        return FESOMC_ECUDA_LC;
    const UnitPlan up = unit_plan(K1p, N4p);
    std::vector<uint16_t> w(up.total / 2, 0);
    const int fan_in[4] = {n->IN, 256, 256, 256}, fan_out[4] = {256, 256, 256, n->OUT};
    for (int i = 0; i < up.n; ++i) {
        const int l = up.layer[i], R = up.rows[i];
        uint16_t *base = w.data() + up.off[i] / 2;
        for (int r = 0; r < R; ++r) {
            const int neuron = up.first_neuron[i] + r;
            if (neuron >= fan_out[l]) continue;   // zero padding of W4
            for (int k = 0; k < fan_in[l]; ++k)
                base[cm_index(R, r, k)] = bf16_bits(p[n->off[l] + (size_t)neuron * fan_in[l] + k]);
        }
    }
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
    if (B < 1) return 0;
    TcParams p{};
    p.IN = n->IN;
    p.OUT = n->OUT;
    p.K1p = k1p_of(n);
    p.N4p = n4p_of(n);
    p.ncol = B;
    p.X = X;
    p.Y = Y;
    p.W = reinterpret_cast<const unsigned char *>(n->wtc);
    const UnitPlan up = unit_plan(p.K1p, p.N4p);
    p.n_units = up.n;
    for (int i = 0; i < up.n; ++i) {
        p.unit_off[i] = up.off[i];
        p.unit_bytes[i] = up.bytes[i];
        p.unit_rows[i] = up.rows[i];
        p.unit_k[i] = up.k[i];
        p.unit_col[i] = up.col[i];
        p.unit_last[i] = up.last[i];
    }
    for (int l = 0, i = 0; l < 4; ++l) {
        p.layer_start[l] = i;
        while (i < up.n && up.layer[i] == l) ++i;
        p.layer_start[l + 1] = i;
    }
    p.b1 = n->params + n->off[0] + (long long)256 * n->IN;
    p.b2 = n->params + n->off[1] + (long long)256 * 256;
    p.b3 = n->params + n->off[2] + (long long)256 * 256;
    p.b4 = n->params + n->off[3] + (long long)n->OUT * 256;
    p.err = n->tc_err;
    const size_t smem = tc_smem(p.IN, &p);
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

size_t lc_tc_smem_bytes(const LcNet *n) { return tc_smem(n->IN, nullptr); }

}  // namespace fesomc
