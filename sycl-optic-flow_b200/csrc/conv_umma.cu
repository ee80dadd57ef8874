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
                                                         int flags, int *err) {
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
        const int yy = pp * d.stride + tap / 3 - 1, xx = pq * d.stride + tap % 3 - 1;
        const bool ok = mval && yy >= 0 && yy < d.H && xx >= 0 && xx < d.W;
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
        const bool relu = flags & 1, f32 = flags & 2;
        const bool vec = d.K % 8 == 0;  // rows of y start on 16-byte boundaries
#pragma unroll 1
        for (int c0 = 0; c0 < NP; c0 += 16) {
            uint32_t r[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
            if (mo >= M) continue;
            float v[16];
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const int col = c0 + j;
                float t = __uint_as_float(r[j]) + (col < d.K ? bias[col] : 0.0f);
                v[j] = relu ? fmaxf(t, 0.0f) : t;
            }
            if (f32) {
                float *o = static_cast<float *>(y) + (size_t)mo * d.K + c0;
#pragma unroll
                for (int j = 0; j < 16; j += 4)
                    if (vec && c0 + j + 3 < d.K)
                        *reinterpret_cast<float4 *>(o + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
                    else
                        for (int e = 0; e < 4; e++)
                            if (c0 + j + e < d.K) o[j + e] = v[j + e];
            } else {
                __nv_bfloat16 *o = static_cast<__nv_bfloat16 *>(y) + (size_t)mo * d.K + c0;
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
                 void *y, int flags, int *err, cudaStream_t st) {
    constexpr int smem = kUmStages * um_stage_bytes<NP, CK>();
    OF_CUDA(cudaFuncSetAttribute(k_conv_fwd_umma<NP, CK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 smem));
    const int M = d.N * d.P * d.Q;
    k_conv_fwd_umma<NP, CK><<<div_up(M, kUmBM), kUmNT, smem, st>>>(d, x, w, bias, y, flags, err);
}

template <int CK>
bool dispatch_np(int np, const ConvDims &d, const __nv_bfloat16 *x, const __nv_bfloat16 *w,
                 const float *bias, void *y, int flags, int *err, cudaStream_t st) {
    switch (np) {
        case 16: launch_umma<16, CK>(d, x, w, bias, y, flags, err, st); return true;
        case 32: launch_umma<32, CK>(d, x, w, bias, y, flags, err, st); return true;
        case 48: launch_umma<48, CK>(d, x, w, bias, y, flags, err, st); return true;
        case 64: launch_umma<64, CK>(d, x, w, bias, y, flags, err, st); return true;
        case 96: launch_umma<96, CK>(d, x, w, bias, y, flags, err, st); return true;
        case 128: launch_umma<128, CK>(d, x, w, bias, y, flags, err, st); return true;
        default: return false;
    }
}

}  // namespace

bool conv_forward_umma(const ConvDims &d, const __nv_bfloat16 *x, const __nv_bfloat16 *w,
                       const float *bias, void *y, bool y_f32, bool relu, int *err, cudaStream_t st) {
    if (d.C % 16 != 0 || d.K > 128 || d.K < 1) return false;
    // 16-byte cp.async sources and vector stores
    const auto a16 = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
    if (!a16(x) || !a16(w) || !a16(y)) return false;
    const int np = (d.K + 15) / 16 * 16;
    const int flags = (relu ? 1 : 0) | (y_f32 ? 2 : 0);
    if (d.C % 32 == 0) return dispatch_np<32>(np, d, x, w, bias, y, flags, err, st);
    return dispatch_np<16>(np, d, x, w, bias, y, flags, err, st);
}

}  // namespace oflow
