// Forward 3x3 convolution (pad 1, stride 1 or 2) of the warm-start network on
// the 5th-generation tensor cores: an implicit GEMM with tcgen05.mma (BF16 in,
// FP32 accumulate in tensor memory).
//
//   out[m][k] = bias[k] + sum_{tap, c} x[n][p*st+r-1][q*st+s-1][c] * w[k][tap][c]
//   m = (n, p, q) flattened (NHWC), tap = 3r + s
//
// One CTA (4 warps) owns 128 consecutive output pixels and all NP (= K padded
// to a multiple of 16) output channels.  The reduction runs over stages of one
// tap x CK channels: every thread gathers its pixel's CK channels of the tap
// (16-byte cp.async, zero-filled outside the image) and a share of the
// weights into shared memory in the no-swizzle K-major layout of the UMMA
// descriptors (8-row x 16-byte core matrices); thread 0 then issues CK/16
// MMAs of 128 x NP x 16 and commits them to the stage's mbarrier.  Four stage
// buffers with a prefetch distance of two let the gathers of stage s+2 and the
// MMAs of stage s+1 run while stage s computes.  The epilogue reads the
// accumulator back with tcgen05.ld (warp w holds TMEM lanes 32w..32w+31, one
// pixel per thread), adds the bias, applies the ReLU and stores bf16 or f32.
//
// Every wait on an mbarrier is bounded (kWaitNs of %globaltimer); when one
// gives up, the kernel sets *err, waits (bounded) for its own copies, frees
// its tensor memory and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "cnn.cuh"
#include "common.cuh"
#include "internal.hpp"
#include "ptx.cuh"

namespace oflow {
namespace {

constexpr int kUmBM = 128;       // output pixels per CTA (UMMA M)
constexpr int kUmNT = 128;       // threads per CTA
constexpr int kUmStages = 4;     // shared-memory stage buffers
constexpr int kUmAhead = 2;      // stages gathered ahead of the one being multiplied

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, bool valid) {
    const int n = valid ? 16 : 0;  // 0 bytes read: the destination is zero-filled
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}

// Shared-memory matrix descriptor, no swizzle, K-major: start address, LBO =
// byte distance between core matrices along K, SBO = byte distance between
// 8-row groups along M/N (all in 16-byte units), version 1 (bits 46-47).
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: D f32 (bits 4-5 = 1), A and B bf16
// (bits 7-9 = 1, 10-12 = 1), both K-major, N/8 at bit 17, M/16 at bit 24.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
        "[%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

template <int NP> __host__ __device__ constexpr uint32_t tmem_cols() { return NP <= 32 ? 32 : NP <= 64 ? 64 : NP <= 128 ? 128 : 256; }

template <int NP, int CK> __host__ __device__ constexpr int um_stage_bytes() { return (kUmBM + NP) * CK * 2; }

template <int NP, int CK>
__global__ void __launch_bounds__(kUmNT) k_conv_fwd_umma(ConvDims d, const __nv_bfloat16 *__restrict__ x,
                                                         const __nv_bfloat16 *__restrict__ w,
                                                         const float *__restrict__ bias, void *y,
                                                         int flags, int ldy, int *err) {
    static_assert(NP % 16 == 0 && NP >= 16 && NP <= 256, "UMMA M=128 needs N = 16..256, step 16");
    static_assert(CK == 16 || CK == 32, "stage depth is 16 or 32 channels");
    constexpr int A_BYTES = kUmBM * CK * 2;
    constexpr int STAGE = um_stage_bytes<NP, CK>();
    constexpr uint32_t TCOLS = tmem_cols<NP>();
    constexpr uint32_t IDESC = umma_idesc_bf16(kUmBM, NP);
    extern __shared__ __align__(1024) uint8_t um_smem[];
    __shared__ __align__(8) uint64_t mbar[kUmStages];
    __shared__ uint32_t tmem_base;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int M = d.N * d.P * d.Q;
    const int m0 = blockIdx.x * kUmBM;
    const int nchunk = d.C / CK;
    const int nst = 9 * nchunk;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_u32(&tmem_base)),
                     "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 0) {
        for (int i = 0; i < kUmStages; i++) mbar_init(smem_u32(&mbar[i]), 1);
        fence_mbar_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;

    // this thread gathers output pixel m0 + tid
    const int m = m0 + tid;
    const bool mval = m < M;
    int pn = 0, pp = 0, pq = 0;
    if (mval) {
        pq = m % d.Q;
        const int t = m / d.Q;
        pp = t % d.P;
        pn = t / d.P;
    }
    const uint32_t sbase = smem_u32(um_smem);

    auto gather = [&](int s) {
        const int buf = s % kUmStages;
        const int tap = s / nchunk, c0 = (s % nchunk) * CK;
        int yy, xx;
        bool ok;
        if (d.stride > 0) {
            yy = pp * d.stride + tap / 3 - 1;
            xx = pq * d.stride + tap % 3 - 1;
            ok = mval && yy >= 0 && yy < d.H && xx >= 0 && xx < d.W;
        } else {
            // input dilated by 2 (the backward-data product of a stride-2
            // layer): output (p, q) reads input ((p + r - 1)/2, (q + s - 1)/2)
            // where both are whole
            const int y2 = pp + tap / 3 - 1, x2 = pq + tap % 3 - 1;
            yy = y2 >> 1;
            xx = x2 >> 1;
            ok = mval && ((y2 | x2) & 1) == 0 && y2 >= 0 && x2 >= 0 && yy < d.H && xx < d.W;
        }
        const __nv_bfloat16 *src = ok ? x + (((size_t)pn * d.H + yy) * d.W + xx) * d.C + c0 : x;
        const uint32_t a = sbase + buf * STAGE;
#pragma unroll
        for (int kc = 0; kc < CK / 8; kc++) cp_async16(a + kc * (kUmBM * 16) + tid * 16, src + kc * 8, ok);
        const uint32_t b = a + A_BYTES;
        for (int e = tid; e < NP * (CK / 8); e += kUmNT) {
            const int n = e % NP, kc = e / NP;
            const bool okb = n < d.K;
            const __nv_bfloat16 *ws = okb ? w + ((size_t)n * 9 + tap) * d.C + c0 + kc * 8 : w;
            cp_async16(b + kc * (NP * 16) + n * 16, ws, okb);
        }
    };

    // one cp.async group per stage (empty past the last), so waiting until
    // kUmAhead groups are pending means stage s has landed
    bool timed_out = false;
#pragma unroll 1
    for (int s = 0; s < kUmAhead; s++) {
        if (s < nst) gather(s);
        cp_async_commit();
    }
#pragma unroll 1
    for (int s = 0; s < nst; s++) {
        const int sl = s + kUmAhead;
        if (sl < nst) {
            // buffer sl % 4 last held stage sl - 4 = s - 2, committed two stages ago
            if (sl >= kUmStages && !timed_out) {
                const int so = sl - kUmStages;
                if (!mbar_wait_bounded(smem_u32(&mbar[so % kUmStages]), (so / kUmStages) & 1))
                    timed_out = true;
            }
            gather(sl);
        }
        cp_async_commit();  // one group per stage (possibly empty)
        cp_async_wait<kUmAhead>();
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const int buf = s % kUmStages;
            const uint32_t a = sbase + buf * STAGE, b = a + A_BYTES;
#pragma unroll
            for (int j = 0; j < CK / 16; j++) {
                const uint64_t ad = umma_desc(a + 2 * j * (kUmBM * 16), kUmBM * 16, 128);
                const uint64_t bd = umma_desc(b + 2 * j * (NP * 16), NP * 16, 128);
                umma_bf16(tmem, ad, bd, IDESC, (s > 0 || j > 0) ? 1u : 0u);
            }
            umma_commit(smem_u32(&mbar[buf]));
        }
    }
    // the last commit tracks every MMA of this CTA
    {
        const int sL = nst - 1;
        if (!timed_out && !mbar_wait_bounded(smem_u32(&mbar[sL % kUmStages]), (sL / kUmStages) & 1))
            timed_out = true;
    }
    cp_async_wait<0>();
    // block-uniform from here: tcgen05.ld is warp-collective
    timed_out = __syncthreads_or(timed_out);
    if (timed_out && tid == 0) atomicOr(err, 1);
    tc_fence_after();
    if (!timed_out) {
        const int mo = m0 + warp * 32 + lane;
        const bool relu = flags & 1, f32 = flags & 2, accum = flags & 4;
        const int ld = ldy > 0 ? ldy : d.K;  // elements between output rows
        const bool vec = d.K % 8 == 0 && ld % 8 == 0;  // rows of y start on 16-byte boundaries
#pragma unroll 1
        for (int c0 = 0; c0 < NP; c0 += 16) {
            uint32_t r[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
            if (mo >= M) continue;
            float v[16];
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const int col = c0 + j;
                float t = __uint_as_float(r[j]) + ((bias && col < d.K) ? bias[col] : 0.0f);
                v[j] = relu ? fmaxf(t, 0.0f) : t;
            }
            if (f32) {
                float *o = static_cast<float *>(y) + (size_t)mo * ld + c0;
                if (accum) {  // each output element belongs to one thread
#pragma unroll
                    for (int j = 0; j < 16; j++)
                        if (c0 + j < d.K) o[j] += v[j];
                    continue;
                }
#pragma unroll
                for (int j = 0; j < 16; j += 4)
                    if (vec && c0 + j + 3 < d.K)
                        *reinterpret_cast<float4 *>(o + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
                    else
                        for (int e = 0; e < 4; e++)
                            if (c0 + j + e < d.K) o[j + e] = v[j + e];
            } else {
                __nv_bfloat16 *o = static_cast<__nv_bfloat16 *>(y) + (size_t)mo * ld + c0;
#pragma unroll
                for (int j = 0; j < 16; j += 8) {
                    if (vec && c0 + j + 7 < d.K) {
                        uint4 pk;
                        __nv_bfloat162 h0 = __floats2bfloat162_rn(v[j], v[j + 1]);
                        __nv_bfloat162 h1 = __floats2bfloat162_rn(v[j + 2], v[j + 3]);
                        __nv_bfloat162 h2 = __floats2bfloat162_rn(v[j + 4], v[j + 5]);
                        __nv_bfloat162 h3 = __floats2bfloat162_rn(v[j + 6], v[j + 7]);
                        pk.x = *reinterpret_cast<uint32_t *>(&h0);
                        pk.y = *reinterpret_cast<uint32_t *>(&h1);
                        pk.z = *reinterpret_cast<uint32_t *>(&h2);
                        pk.w = *reinterpret_cast<uint32_t *>(&h3);
                        *reinterpret_cast<uint4 *>(o + j) = pk;
                    } else {
                        for (int e = 0; e < 8; e++)
                            if (c0 + j + e < d.K) o[j + e] = __float2bfloat16(v[j + e]);
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS)
                     : "memory");
}

template <int NP, int CK>
void launch_umma(const ConvDims &d, const __nv_bfloat16 *x, const __nv_bfloat16 *w, const float *bias,
                 void *y, int flags, int ldy, int *err, cudaStream_t st) {
    constexpr int smem = kUmStages * um_stage_bytes<NP, CK>();
    OF_CUDA(cudaFuncSetAttribute(k_conv_fwd_umma<NP, CK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 smem));
    const int M = d.N * d.P * d.Q;
    k_conv_fwd_umma<NP, CK><<<div_up(M, kUmBM), kUmNT, smem, st>>>(d, x, w, bias, y, flags, ldy, err);
}

template <int CK>
bool dispatch_np(int np, const ConvDims &d, const __nv_bfloat16 *x, const __nv_bfloat16 *w,
                 const float *bias, void *y, int flags, int ldy, int *err, cudaStream_t st) {
    switch (np) {
        case 16: launch_umma<16, CK>(d, x, w, bias, y, flags, ldy, err, st); return true;
        case 32: launch_umma<32, CK>(d, x, w, bias, y, flags, ldy, err, st); return true;
        case 48: launch_umma<48, CK>(d, x, w, bias, y, flags, ldy, err, st); return true;
        case 64: launch_umma<64, CK>(d, x, w, bias, y, flags, ldy, err, st); return true;
        case 96: launch_umma<96, CK>(d, x, w, bias, y, flags, ldy, err, st); return true;
        case 128: launch_umma<128, CK>(d, x, w, bias, y, flags, ldy, err, st); return true;
        default: return false;
    }
}

// Backward-weight product on the tensor cores:
//   gw[k][tap][c] = sum_m x[pixel(m, tap)][c] * g[m][k]
// as D = A B with the rows of D the (tap, c) pairs of the layer (9C rows, in
// 128-row UMMA tiles, row = tap * C + c), its columns the output channels k
// (K rounded up to 16 = KP) and the reduction over output pixels m, 32 per
// stage.  Both operands are read in the layout they have in memory and
// staged MN-major (no swizzle): a core matrix is 8 reduction rows (pixels) of
// 16 bytes, each 16 bytes being 8 consecutive (tap, c) rows of A -- the
// channels c..c+7 of one input pixel -- or 8 consecutive output channels of B
// -- g[m][k..k+7].  So every gather is one 16-byte cp.async of NHWC memory,
// with no transposition.  In a stage, core matrices along the reduction are
// 128 bytes apart (LBO) and groups of 8 rows 512 bytes apart (SBO); tile t of
// A starts t * 8 KB into the stage.  A CTA owns up to kWgMT tiles of rows
// (gridDim.x runs over groups of tiles), shares each stage's gradient tile
// between them, reduces a range of pixels (gridDim.y splits the pixels) and
// adds its rows to gw with atomics.  Pipeline, commits and bounded waits as in
// the forward kernel.
constexpr int kWgMT = 4;       // row tiles a CTA at most
constexpr int kWgPix = 32;     // pixels a stage
constexpr int kWgTile = kUmBM * kWgPix * 2;  // bytes of one row tile a stage

template <int KP>
__global__ void __launch_bounds__(kUmNT) k_conv_wgrad_mn(ConvDims d, const __nv_bfloat16 *__restrict__ gb,
                                                         const __nv_bfloat16 *__restrict__ x, float *gw,
                                                         int ntg, int pix_per_cta, uint32_t tcols, int *err) {
    static_assert(KP % 16 == 0 && KP >= 16 && KP <= 128, "N = 16..128, step 16");
    constexpr uint32_t IDESC = umma_idesc_bf16(kUmBM, KP) | (1u << 15) | (1u << 16);  // A, B MN-major
    constexpr int B_BYTES = KP * kWgPix * 2;
    extern __shared__ __align__(1024) uint8_t um_smem[];
    __shared__ __align__(8) uint64_t mbar[kUmStages];
    __shared__ uint32_t tmem_base;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int M = d.N * d.P * d.Q;
    const int rows = 9 * d.C;
    const int tiles = div_up(rows, kUmBM);
    const int t0 = blockIdx.x * ntg;                 // first row tile of this CTA
    const int nt = imin(ntg, tiles - t0);            // row tiles of this CTA
    const int stage_bytes = ntg * kWgTile + B_BYTES;
    const int m_lo = blockIdx.y * pix_per_cta;
    const int m_hi = imin(M, m_lo + pix_per_cta);
    const int nst = m_hi > m_lo ? div_up(m_hi - m_lo, kWgPix) : 0;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_u32(&tmem_base)),
                     "r"(tcols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 0) {
        for (int i = 0; i < kUmStages; i++) mbar_init(smem_u32(&mbar[i]), 1);
        fence_mbar_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    const uint32_t sbase = smem_u32(um_smem);

    // This thread gathers pixel j = 8 warp + (lane & 7) of every stage, for the
    // 8-row groups g = 4 i + (lane >> 3) of A and the channel groups
    // kg = 4 i + (lane >> 3) of B.  Row group g: tap, first channel, and the
    // element offset of its 8 channels from the tap's centre pixel.
    const int j = warp * 8 + (lane & 7), gs = lane >> 3;
    int toff[kWgMT * 4], tap_rs[kWgMT * 4];
#pragma unroll
    for (int i = 0; i < kWgMT * 4; i++) {
        const int R = (t0 * 16 + 4 * i + gs) * 8;  // first row of the group
        if (i < nt * 4 && R < rows) {
            const int tap = R / d.C, c = R % d.C, r = tap / 3, sx = tap % 3;
            toff[i] = (r * d.W + sx) * d.C + c;
            tap_rs[i] = r | (sx << 2);
        } else {
            toff[i] = 0;
            tap_rs[i] = -1;
        }
    }
    const uint32_t jo = (uint32_t)((j >> 3) * 128 + (j & 7) * 16);

    auto gather = [&](int s) {
        const uint32_t a = sbase + (s % kUmStages) * stage_bytes;
        const uint32_t b = a + ntg * kWgTile;
        const int m = m_lo + s * kWgPix + j;
        const bool mv = m < m_hi;
        int y0 = 0, x0 = 0;
        long long pbase = 0;
        if (mv) {
            const int q = m % d.Q, t = m / d.Q, p = t % d.P, n = t / d.P;
            y0 = p * d.stride - 1;
            x0 = q * d.stride - 1;
            pbase = (((long long)n * d.H + y0) * d.W + x0) * d.C;
        }
#pragma unroll
        for (int i = 0; i < kWgMT * 4; i++) {
            if (i < nt * 4) {
                const int rs = tap_rs[i];
                const bool ok = mv && rs >= 0 && (unsigned)(y0 + (rs & 3)) < (unsigned)d.H &&
                                (unsigned)(x0 + (rs >> 2)) < (unsigned)d.W;
                cp_async16(a + (uint32_t)(4 * i + gs) * 512 + jo, ok ? x + pbase + toff[i] : x, ok);
            }
        }
#pragma unroll
        for (int i = 0; i < (KP / 8 + 3) / 4; i++) {
            const int kg = 4 * i + gs;
            if (kg < KP / 8) {
                const bool ok = mv && kg * 8 < d.K;
                cp_async16(b + (uint32_t)kg * 512 + jo, ok ? gb + (size_t)m * d.K + kg * 8 : gb, ok);
            }
        }
    };

    // one cp.async group per stage (empty past the last), so waiting until
    // kUmAhead groups are pending means stage s has landed
    bool timed_out = false;
#pragma unroll 1
    for (int s = 0; s < kUmAhead; s++) {
        if (s < nst) gather(s);
        cp_async_commit();
    }
#pragma unroll 1
    for (int s = 0; s < nst; s++) {
        const int sl = s + kUmAhead;
        if (sl < nst) {
            // buffer sl % 4 last held stage sl - 4 = s - 2, committed two stages ago
            if (sl >= kUmStages && !timed_out) {
                const int so = sl - kUmStages;
                if (!mbar_wait_bounded(smem_u32(&mbar[so % kUmStages]), (so / kUmStages) & 1))
                    timed_out = true;
            }
            gather(sl);
        }
        cp_async_commit();
        cp_async_wait<kUmAhead>();
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const int buf = s % kUmStages;
            const uint32_t a = sbase + buf * stage_bytes, b = a + ntg * kWgTile;
#pragma unroll 1
            for (int t = 0; t < nt; t++) {
#pragma unroll
                for (int h = 0; h < kWgPix / 16; h++) {
                    const uint64_t ad = umma_desc(a + t * kWgTile + h * 256, 128, 512);
                    const uint64_t bd = umma_desc(b + h * 256, 128, 512);
                    umma_bf16(tmem + (uint32_t)(t * KP), ad, bd, IDESC, (s > 0 || h > 0) ? 1u : 0u);
                }
            }
            umma_commit(smem_u32(&mbar[buf]));
        }
    }
    if (nst > 0) {
        const int sL = nst - 1;
        if (!timed_out && !mbar_wait_bounded(smem_u32(&mbar[sL % kUmStages]), (sL / kUmStages) & 1))
            timed_out = true;
    }
    cp_async_wait<0>();
    timed_out = __syncthreads_or(timed_out);
    if (timed_out && tid == 0) atomicOr(err, 1);
    tc_fence_after();
    if (!timed_out && nst > 0) {
#pragma unroll 1
        for (int t = 0; t < nt; t++) {
            const int R = (t0 + t) * kUmBM + warp * 32 + lane;  // TMEM lane = row of D
            const bool rv = R < rows;
            const int tap = rv ? R / d.C : 0, c = rv ? R % d.C : 0;
#pragma unroll 1
            for (int cc = 0; cc < KP; cc += 16) {
                uint32_t r[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(t * KP + cc), r);
                if (!rv) continue;
#pragma unroll
                for (int e = 0; e < 16; e++)
                    if (cc + e < d.K) atomicAdd(gw + ((size_t)(cc + e) * 9 + tap) * d.C + c, __uint_as_float(r[e]));
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(tcols)
                     : "memory");
}

template <int KP>
void launch_wgrad(const ConvDims &d, const __nv_bfloat16 *gb, const __nv_bfloat16 *x, float *gw,
                  int *err, cudaStream_t st) {
    const int M = d.N * d.P * d.Q;
    if (M <= 0) return;
    const int tiles = div_up(9 * d.C, kUmBM);
    const int groups = div_up(tiles, kWgMT);
    const int ntg = div_up(tiles, groups);  // row tiles a CTA, balanced over the groups
    const int smem = kUmStages * (ntg * kWgTile + KP * kWgPix * 2);
    uint32_t tcols = 32;
    while (tcols < (uint32_t)(ntg * KP)) tcols <<= 1;
    OF_CUDA(cudaFuncSetAttribute(k_conv_wgrad_mn<KP>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    // CTAs an SM holds by shared memory and tensor memory; one wave of them
    const int occ = imax(1, imin((227 * 1024) / (smem + 1024), (int)(512 / tcols)));
    const int splits = imax(1, imin(div_up(M, kWgPix), div_up(kNumSMs * occ, groups)));
    const int per = div_up(div_up(M, splits), kWgPix) * kWgPix;
    k_conv_wgrad_mn<KP><<<dim3(groups, div_up(M, per)), kUmNT, smem, st>>>(d, gb, x, gw, ntg, per, tcols, err);
}

// bf16 copy of the output gradient, zero where the layer's ReLU was inactive
// (the same masking and rounding the mma.sync backward applies on its gather)
__global__ void k_mask_bf16(const float *__restrict__ g, const __nv_bfloat16 *__restrict__ yact,
                            __nv_bfloat16 *out, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        float v = g[i];
        if (yact && !(__bfloat162float(yact[i]) > 0.0f)) v = 0.0f;
        out[i] = __float2bfloat16(v);
    }
}

// The same masked bf16 copy fused with the bias gradient's first stage, for
// K % 4 == 0 (K <= 128): block b covers the gradient rows (output pixels)
// [b * rpb, (b + 1) * rpb); a thread keeps four adjacent channels (one float4
// of a row) and walks R = 256 / (K / 4) rows apart, so each step of the block
// reads whole rows.  The per-thread sums then go, in a fixed order, to one
// partial sum per channel and block: partial[b * K + k].
constexpr int kBiasBlocks = 4 * kNumSMs;
constexpr int kBiasFinalNT = 256;

// Scratch of the backward products, in bytes from its start: the masked bf16
// gradient, the rotated weights (each rounded up to 64 elements, 128-byte
// aligned), then the bias partial sums (kBiasBlocks x K floats).
size_t bwd_scratch_part(const ConvDims &d) {
    const size_t kp = (size_t)(d.K + 15) / 16 * 16;  // gradient channels padded to 16
    const size_t g = (size_t)d.N * d.P * d.Q * kp, wt = kp * 9 * d.C;
    return ((g + 63) / 64 * 64 + (wt + 63) / 64 * 64) * sizeof(__nv_bfloat16);
}

__global__ void __launch_bounds__(256) k_mask_bias(const float *__restrict__ g,
                                                   const __nv_bfloat16 *__restrict__ yact,
                                                   __nv_bfloat16 *__restrict__ out, int M, int K,
                                                   int rpb, float *__restrict__ partial) {
    __shared__ float4 sh[256];
    const int Q = K >> 2, R = 256 / Q, t = threadIdx.x;
    const int q = t % Q, ro = t / Q;
    float4 s = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (ro < R) {
        const int r0 = blockIdx.x * rpb, r1 = imin(r0 + rpb, M);
        for (int r = r0 + ro; r < r1; r += R) {
            const size_t i = (size_t)r * K + 4 * q;
            float4 v = __ldg(reinterpret_cast<const float4 *>(g + i));
            if (yact) {
                const uint2 a = __ldg(reinterpret_cast<const uint2 *>(yact + i));
                const __nv_bfloat162 a01 = *reinterpret_cast<const __nv_bfloat162 *>(&a.x);
                const __nv_bfloat162 a23 = *reinterpret_cast<const __nv_bfloat162 *>(&a.y);
                if (!(__low2float(a01) > 0.0f)) v.x = 0.0f;
                if (!(__high2float(a01) > 0.0f)) v.y = 0.0f;
                if (!(__low2float(a23) > 0.0f)) v.z = 0.0f;
                if (!(__high2float(a23) > 0.0f)) v.w = 0.0f;
            }
            s.x += v.x;
            s.y += v.y;
            s.z += v.z;
            s.w += v.w;
            const __nv_bfloat162 o01 = __floats2bfloat162_rn(v.x, v.y);
            const __nv_bfloat162 o23 = __floats2bfloat162_rn(v.z, v.w);
            uint2 o;
            o.x = *reinterpret_cast<const uint32_t *>(&o01);
            o.y = *reinterpret_cast<const uint32_t *>(&o23);
            *reinterpret_cast<uint2 *>(out + i) = o;
        }
    }
    sh[t] = s;
    __syncthreads();
    if (t < K) {
        const int qq = t >> 2, e = t & 3;
        float acc = 0.0f;
        for (int j = 0; j < R; j++) {
            const float4 w = sh[j * Q + qq];
            acc += e == 0 ? w.x : e == 1 ? w.y : e == 2 ? w.z : w.w;
        }
        partial[(size_t)blockIdx.x * K + t] = acc;
    }
}

// gb[k] = the sum of the nb partial sums of channel k, one block a channel:
// thread t adds blocks t, t + NT, ... in order, then a fixed tree adds the
// threads' sums.
__global__ void __launch_bounds__(kBiasFinalNT) k_bias_final(const float *__restrict__ partial,
                                                             int nb, int K, float *gb) {
    __shared__ double scratch[kBiasFinalNT / 32];
    const int k = blockIdx.x;
    float acc = 0.0f;
    for (int b = threadIdx.x; b < nb; b += kBiasFinalNT) acc += __ldg(partial + (size_t)b * K + k);
    const double r = block_sum_double<kBiasFinalNT>((double)acc, scratch);
    if (threadIdx.x == 0) gb[k] = (float)r;
}

// wt[c][tap][k] = w[k][8 - tap][c]: the weights of the backward-data product
// seen as a forward convolution (rotated taps, input and output channels
// exchanged), with Kp >= K input channels (zero for k >= K)
__global__ void k_flip_weights(const __nv_bfloat16 *__restrict__ w, int K, int Kp, int C,
                               __nv_bfloat16 *wt) {
    const int n = Kp * 9 * C;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int k = i % Kp, tap = (i / Kp) % 9, c = i / (9 * Kp);
        wt[i] = k < K ? w[((size_t)k * 9 + (8 - tap)) * C + c] : __float2bfloat16(0.0f);
    }
}

// masked bf16 gradient with its K channels padded to Kp (zero): out[m][k]
__global__ void k_mask_pad_bf16(const float *__restrict__ g, const __nv_bfloat16 *__restrict__ yact,
                                int M, int K, int Kp, __nv_bfloat16 *out) {
    const size_t n = (size_t)M * Kp;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t m = i / Kp;
        const int k = (int)(i - m * Kp);
        float v = 0.0f;
        if (k < K) {
            v = g[m * K + k];
            if (yact && !(__bfloat162float(yact[m * K + k]) > 0.0f)) v = 0.0f;
        }
        out[i] = __float2bfloat16(v);
    }
}

}  // namespace

bool conv_forward_umma(const ConvDims &d, const __nv_bfloat16 *x, const __nv_bfloat16 *w,
                       const float *bias, void *y, bool y_f32, bool relu, int *err, cudaStream_t st,
                       int ldy, bool accumulate) {
    if (d.C % 16 != 0 || d.K > 128 || d.K < 1) return false;
    if (accumulate && !y_f32) return false;
    // 16-byte cp.async sources and vector stores
    const auto a16 = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
    if (!a16(x) || !a16(w) || !a16(y)) return false;
    const int np = (d.K + 15) / 16 * 16;
    const int flags = (relu ? 1 : 0) | (y_f32 ? 2 : 0) | (accumulate ? 4 : 0);
    if (d.C % 32 == 0) return dispatch_np<32>(np, d, x, w, bias, y, flags, ldy, err, st);
    return dispatch_np<16>(np, d, x, w, bias, y, flags, ldy, err, st);
}

bool conv_backward_weight_umma(const ConvDims &d, const float *g, const __nv_bfloat16 *y_act,
                               const __nv_bfloat16 *x, float *gw, float *gb, void *scratch,
                               int *err, cudaStream_t st) {
    if (d.K > 128 || d.K % 8 != 0 || d.C % 16 != 0) return false;
    if ((reinterpret_cast<uintptr_t>(x) & 15u) != 0 || (reinterpret_cast<uintptr_t>(scratch) & 15u) != 0)
        return false;
    const size_t ng = (size_t)d.N * d.P * d.Q * d.K;
    __nv_bfloat16 *gbf = static_cast<__nv_bfloat16 *>(scratch);
    // the masked bf16 copy and the bias gradient in one pass over g where the
    // channels split into float4 quads
    const int M = d.N * d.P * d.Q;
    const bool fused = M > 0 && d.K % 4 == 0 && (reinterpret_cast<uintptr_t>(g) & 15u) == 0 &&
                       (y_act == nullptr || (reinterpret_cast<uintptr_t>(y_act) & 7u) == 0);
    if (fused) {
        const int R = 256 / (d.K / 4);
        const int rpb = div_up(div_up(M, imin(kBiasBlocks, imax(1, div_up(M, 4 * R)))), R) * R;
        const int nb = div_up(M, rpb);
        float *part = reinterpret_cast<float *>(static_cast<char *>(scratch) + bwd_scratch_part(d));
        k_mask_bias<<<nb, 256, 0, st>>>(g, y_act, gbf, M, d.K, rpb, part);
        k_bias_final<<<d.K, kBiasFinalNT, 0, st>>>(part, nb, d.K, gb);
    } else {
        k_mask_bf16<<<imin((int)((ng + 255) / 256), 4096), 256, 0, st>>>(g, y_act, gbf, ng);
    }
    OF_CUDA(cudaMemsetAsync(gw, 0, sizeof(float) * (size_t)d.K * 9 * d.C, st));
    switch ((d.K + 15) / 16 * 16) {
        case 16: launch_wgrad<16>(d, gbf, x, gw, err, st); break;
        case 32: launch_wgrad<32>(d, gbf, x, gw, err, st); break;
        case 48: launch_wgrad<48>(d, gbf, x, gw, err, st); break;
        case 64: launch_wgrad<64>(d, gbf, x, gw, err, st); break;
        case 80: launch_wgrad<80>(d, gbf, x, gw, err, st); break;
        case 96: launch_wgrad<96>(d, gbf, x, gw, err, st); break;
        case 112: launch_wgrad<112>(d, gbf, x, gw, err, st); break;
        default: launch_wgrad<128>(d, gbf, x, gw, err, st); break;
    }
    if (!fused) conv_bias_grad(d, g, y_act, gb, st);
    return true;
}

size_t conv_backward_data_umma_scratch(const ConvDims &d) {
    return bwd_scratch_part(d) + sizeof(float) * kBiasBlocks * (size_t)d.K;
}

bool conv_backward_data_umma(const ConvDims &d, const float *g, const __nv_bfloat16 *y_act,
                             const __nv_bfloat16 *w, float *gin, bool accumulate, void *scratch,
                             int *err, cudaStream_t st, bool g_masked) {
    if (d.K % 8 != 0 || d.C % 16 != 0) return false;
    if ((reinterpret_cast<uintptr_t>(gin) & 15u) != 0) return false;
    // the gradient's channels are the product's input channels: padded to a
    // multiple of 16 (zero channels, zero weights) where K is not one
    const int Kp = (d.K + 15) / 16 * 16;
    const int M = d.N * d.P * d.Q;
    const size_t ng = (size_t)M * Kp;
    __nv_bfloat16 *gb = static_cast<__nv_bfloat16 *>(scratch);
    __nv_bfloat16 *wt = gb + (ng + 63) / 64 * 64;  // 128-byte aligned
    if (Kp != d.K)
        k_mask_pad_bf16<<<imin((int)((ng + 255) / 256), 4096), 256, 0, st>>>(g, y_act, M, d.K, Kp, gb);
    else if (!g_masked)
        k_mask_bf16<<<imin((int)((ng + 255) / 256), 4096), 256, 0, st>>>(g, y_act, gb, ng);
    k_flip_weights<<<imin(div_up(Kp * 9 * d.C, 256), 1024), 256, 0, st>>>(w, d.K, Kp, d.C, wt);
    // the product as a forward convolution over the output gradient: input
    // (N, P, Q, Kp), output (N, H, W, C); stride 2 layers read a dilated input
    ConvDims t{d.N, d.P, d.Q, Kp, d.H, d.W, 0, d.stride == 1 ? 1 : -2};
    for (int c0 = 0; c0 < d.C; c0 += 128) {  // at most 128 output channels a launch
        t.K = imin(128, d.C - c0);
        if (!conv_forward_umma(t, gb, wt + (size_t)c0 * 9 * Kp, nullptr, gin + c0, true, false, err,
                               st, d.C, accumulate))
            return false;
    }
    return true;
}

}  // namespace oflow
