// Horn-Schunck on B200: kernels and the batched plan.  Restates
// src/hs/cuda/flow.cu:112-208 and src/hs/cuda/kernels/*.cuh with the
// semantics those kernels are written for (bilinear clamp-to-edge warp and
// upscale, clamped derivative taps, every pixel written); the arithmetic
// contract is in common.cuh.
//
// Layout per pair b (N = w*h at the finest level, levels packed):
//   raw[b][2] staged frames, pyr_l[b][2] float pyramid (finest = nlevels-1),
//   D[b] float4 (Ix, Iy, Iz, Ix^2+Iy^2+alpha), dU0/dU1[b] float2 ping-pong
//   increments, Ua/Ub[b] float2 flow (alternating per level), out[2][b].
// All ping-pong parities are known on the host, so the schedule is static and
// captured into one CUDA graph.
//
// The Jacobi sweeps are temporally blocked: one launch runs up to K sweeps on
// a TW x TH tile held in shared memory with a K-pixel halo; the halo shrinks
// by one pixel per sweep, so after K sweeps the owned tile is exact (clamped
// neighbours at the image border are exact at every sweep).
#include <cstring>

#include "common.cuh"
#include "hs.hpp"
#include "pairio.hpp"
#include "internal.hpp"
#include "ptx.cuh"
#include "tvl1.hpp"

namespace oflow {


// 2x2 box average (downscaleKernel.cuh:27-29), every output pixel written.
__global__ void k_hs_downscale(const float *__restrict__ src, size_t sstride, int w, int h,
                               float *dst, size_t dstride) {
    const int nw = w / 2, nh = h / 2;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= nw || y >= nh) return;
    const float *s = src + (size_t)blockIdx.z * sstride + (size_t)(2 * y) * w + 2 * x;
    dst[(size_t)blockIdx.z * dstride + (size_t)y * nw + x] = 0.25f * (s[0] + s[w] + s[1] + s[w + 1]);
}

__device__ __forceinline__ float hs_deriv5(float m2, float m1, float p1, float p2) {
    float t = m2;
    t -= m1 * 8.0f;
    t += p1 * 8.0f;
    t -= p2;
    t /= 12.0f;
    return t;
}

// Fused warp + derivatives (warpingKernel.cuh:28-44, derivativesKernel.cuh:
// 29-73).  The tile plus a 2-pixel halo is filled with values at clamped
// image coordinates, so a derivative tap at offset k reads the clamped
// neighbour directly.
constexpr int kDTW = 32, kDTH = 8;
__global__ void __launch_bounds__(kDTW *kDTH) k_hs_warp_deriv(
    const float *__restrict__ pyr, size_t lp, int w, int h, const float2 *__restrict__ U,
    size_t ustride, int zero_flow, float alpha, float4 *D, size_t dstride) {
    constexpr int RW = kDTW + 4, RH = kDTH + 4;
    __shared__ float s0[RH * RW], s1[RH * RW];
    const int b = blockIdx.z;
    const float *I0 = pyr + (size_t)(2 * b) * lp;
    const float *I1 = pyr + (size_t)(2 * b + 1) * lp;
    const float2 *Ub = U + (size_t)b * ustride;
    const int x0 = blockIdx.x * kDTW - 2, y0 = blockIdx.y * kDTH - 2;
    const int tid = threadIdx.y * kDTW + threadIdx.x;
    for (int i = tid; i < RW * RH; i += kDTW * kDTH) {
        const int cx = imin(imax(x0 + i % RW, 0), w - 1);
        const int cy = imin(imax(y0 + i / RW, 0), h - 1);
        const size_t p = (size_t)cy * w + cx;
        s0[i] = __ldg(I0 + p);
        const float2 u = zero_flow ? make_float2(0.f, 0.f) : Ub[p];
        s1[i] = bilinear_clamped(I1, w, h, (float)cx + u.x, (float)cy + u.y);
    }
    __syncthreads();
    const int x = blockIdx.x * kDTW + threadIdx.x, y = blockIdx.y * kDTH + threadIdx.y;
    if (x >= w || y >= h) return;
    const int c = (threadIdx.y + 2) * RW + threadIdx.x + 2;
    float t0 = hs_deriv5(s0[c - 2], s0[c - 1], s0[c + 1], s0[c + 2]);
    float t1 = hs_deriv5(s1[c - 2], s1[c - 1], s1[c + 1], s1[c + 2]);
    const float Ix = (t0 + t1) * 0.5f;
    const float Iz = s1[c] - s0[c];
    t0 = hs_deriv5(s0[c - 2 * RW], s0[c - RW], s0[c + RW], s0[c + 2 * RW]);
    t1 = hs_deriv5(s1[c - 2 * RW], s1[c - RW], s1[c + RW], s1[c + 2 * RW]);
    const float Iy = (t0 + t1) * 0.5f;
    const float den = Ix * Ix + Iy * Iy + alpha;
    D[(size_t)b * dstride + (size_t)y * w + x] = make_float4(Ix, Iy, Iz, den);
}

// One Jacobi sweep (solverKernel.cuh:41-153) over cone j of the region:
// neighbour mean of the increments (clamped at the image border), then
// frac = (Ix*su + Iy*sv + Iz) / (Ix^2 + Iy^2 + alpha) and the update, in the
// reference's order.  The division is Markstein's correction from the
// precomputed reciprocal; operands outside its proven range take the IEEE
// division.
template <int RW, int RH, int NT, bool INTERIOR>
__device__ __forceinline__ void hs_sweep(int j, const float2 *src, float2 *dst, const float4 *sD,
                                         const float *sR, int x0, int y0, int w, int h) {
    for_rect<NT>(j, RW - 1 - j, j, RH - 1 - j, [&](int rx, int ry) {
        const int i = ry * RW + rx;
        int l = i - 1, r = i + 1, up = i + RW, dn = i - RW;
        if (!INTERIOR) {
            const int x = x0 + rx, y = y0 + ry;
            if (x < 0 || x >= w || y < 0 || y >= h) return;
            if (x == 0) l = i;
            if (x == w - 1) r = i;
            if (y == h - 1) up = i;
            if (y == 0) dn = i;
        }
        const float2 al = src[l], ar = src[r], au = src[up], ad = src[dn];
        const float su = (al.x + ar.x + au.x + ad.x) * 0.25f;
        const float sv = (al.y + ar.y + au.y + ad.y) * 0.25f;
        const float4 d = sD[i];
        const float p = d.x * su + d.y * sv + d.z;
        float frac = markstein(p, d.w, sR[i]);
        if (!(rcp_in_range(d.w) && markstein_safe(p))) frac = p / d.w;
        dst[i] = make_float2(su - d.x * frac, sv - d.y * frac);
    });
}

// Region loads of k_hs_jacobi by TMA: D as (2w, h, pair) and the incoming
// increments as (w, h, pair), 8-byte elements, zero fill outside the level
// (pixels outside are never read by a sweep).  use = 0: plain loads.
struct HsTma {
    int use;
    int *err;  // set when a bounded wait gives up
    CUtensorMap tD, tIn;
};

// K Jacobi sweeps (solverKernel.cuh:41-153) on a tile with a KH-pixel halo.
// sweeps <= KH.  first: increments start at 0 (flow.cu:168-171).  last: add
// the increment to the flow (AddKernel, addKernel.cuh:28-36) instead of
// storing it.
template <int TW, int TH, int KH, int NT>
__global__ void __launch_bounds__(NT) k_hs_jacobi(const float4 *__restrict__ D, size_t dstride,
                                                  const float2 *__restrict__ dUin,
                                                  float2 *dUout, float2 *U, size_t stride,
                                                  int w, int h, int sweeps, int first, int last,
                                                  const __grid_constant__ HsTma tma) {
    constexpr int RW = TW + 2 * KH, RH = TH + 2 * KH, RN = RW * RH;
    extern __shared__ __align__(128) float4 smem[];
    float4 *sD = smem;                                   // RN
    float2 *sA = reinterpret_cast<float2 *>(sD + RN);    // RN
    float2 *sB = sA + RN;                                // RN
    float *sR = reinterpret_cast<float *>(sB + RN);      // RN
    const int b = blockIdx.z;
    const float4 *Db = D + (size_t)b * dstride;
    const float2 *In = dUin + (size_t)b * stride;
    const int x0 = blockIdx.x * TW - KH, y0 = blockIdx.y * TH - KH;
    const uint32_t sbase = smem_u32(smem);
    if (tma.use && (sbase & 127u) == 0) {
        __shared__ __align__(8) unsigned long long s_bar;
        const uint32_t bar = smem_u32(&s_bar);
        if (threadIdx.x == 0) {
            mbar_init(bar, 1);
            fence_mbar_init();
            mbar_arrive_expect_tx(bar, (uint32_t)RN * (first ? 16u : 24u));
            tma_load_3d(sbase, &tma.tD, 2 * x0, y0, b, bar);
            if (!first) tma_load_3d(sbase + RN * 16, &tma.tIn, x0, y0, b, bar);
        }
        if (first)
            for (int i = threadIdx.x; i < RN; i += NT) sA[i] = make_float2(0.f, 0.f);
        __syncthreads();  // the barrier is initialised before anyone waits on it
        const bool ok = mbar_wait_bounded(bar, 0);
        if (__syncthreads_or(!ok)) {
            // report, let the copies land (bounded), leave; the host drops
            // the plan's results
            if (threadIdx.x == 0) atomicExch(tma.err, 1);
            mbar_wait_bounded(bar, 0);
            return;
        }
    } else {
        for (int i = threadIdx.x; i < RN; i += NT) {
            const int x = x0 + i % RW, y = y0 + i / RW;
            float4 d = make_float4(0.f, 0.f, 0.f, 1.f);
            float2 a = make_float2(0.f, 0.f);
            if (x >= 0 && x < w && y >= 0 && y < h) {
                const size_t p = (size_t)y * w + x;
                d = Db[p];
                if (!first) a = In[p];
            }
            sD[i] = d;
            sA[i] = a;
        }
    }
    __syncthreads();
    // RN(1 / (Ix^2 + Iy^2 + alpha)) per region pixel, constant over the sweeps:
    // the quotient below is then Markstein's exact form (exact_math.cuh)
    for (int i = threadIdx.x; i < RN; i += NT) sR[i] = rcp_near_rn(sD[i].w);
    __syncthreads();
    // Sweep j (1-based) updates [j, RW-1-j] x [j, RH-1-j]: exactly the cells
    // whose values can still reach the owned tile, so no read leaves the
    // region.  A region inside the image with a one-pixel margin takes the
    // path without image-border tests.
    const bool interior = x0 >= 0 && y0 >= 0 && x0 + RW <= w && y0 + RH <= h;
    float2 *src = sA, *dst = sB;
#pragma unroll
    for (int j = 1; j <= KH; j++) {
        if (j > sweeps) break;
        if (interior)
            hs_sweep<RW, RH, NT, true>(j, src, dst, sD, sR, x0, y0, w, h);
        else
            hs_sweep<RW, RH, NT, false>(j, src, dst, sD, sR, x0, y0, w, h);
        __syncthreads();
        float2 *t = src;
        src = dst;
        dst = t;
    }
    for (int i = threadIdx.x; i < TW * TH; i += NT) {
        const int tx = i % TW, ty = i / TW;
        const int x = x0 + KH + tx, y = y0 + KH + ty;
        if (x >= w || y >= h) continue;
        const float2 a = src[(ty + KH) * RW + tx + KH];
        const size_t p = (size_t)b * stride + (size_t)y * w + x;
        if (last) {
            const float2 u = U[p];
            U[p] = make_float2(u.x + a.x, u.y + a.y);
        } else {
            dUout[p] = a;
        }
    }
}

// Flow prolongation (upscaleKernel.cuh:26-40 as a filtering upscale):
// bilinear, clamp-to-edge, centre-aligned, component-wise scale.
__device__ __forceinline__ float2 bilinear2(const float2 *__restrict__ src, int w, int h,
                                            float xf, float yf) {
    xf = fminf(fmaxf(xf, -1.0f), (float)w);
    yf = fminf(fmaxf(yf, -1.0f), (float)h);
    const float x0f = floorf(xf), y0f = floorf(yf);
    const float fx = xf - x0f, fy = yf - y0f;
    const int x0 = (int)x0f, y0 = (int)y0f;
    const int xa = imin(imax(x0, 0), w - 1), xb = imin(imax(x0 + 1, 0), w - 1);
    const int ya = imin(imax(y0, 0), h - 1), yb = imin(imax(y0 + 1, 0), h - 1);
    const float2 v00 = src[(size_t)ya * w + xa], v10 = src[(size_t)ya * w + xb];
    const float2 v01 = src[(size_t)yb * w + xa], v11 = src[(size_t)yb * w + xb];
    const float gx = 1.0f - fx, gy = 1.0f - fy;
    float2 r;
    float top = gx * v00.x + fx * v10.x, bot = gx * v01.x + fx * v11.x;
    r.x = gy * top + fy * bot;
    top = gx * v00.y + fx * v10.y;
    bot = gx * v01.y + fx * v11.y;
    r.y = gy * top + fy * bot;
    return r;
}

__global__ void k_upscale2(const float2 *__restrict__ src, size_t sstride, int w, int h,
                           float2 *dst, size_t dstride, int nw, int nh, float sx, float sy) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= nw || y >= nh) return;
    const float rx = (float)w / (float)nw, ry = (float)h / (float)nh;
    const float fx = ((float)x + 0.5f) * rx - 0.5f;
    const float fy = ((float)y + 0.5f) * ry - 0.5f;
    const float2 r = bilinear2(src + (size_t)blockIdx.z * sstride, w, h, fx, fy);
    dst[(size_t)blockIdx.z * dstride + (size_t)y * nw + x] = make_float2(r.x * sx, r.y * sy);
}

__global__ void k_split2(const float2 *__restrict__ U, size_t stride, int N, float *ou, float *ov,
                         int B) {
    const int b = blockIdx.y;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const float2 u = U[(size_t)b * stride + i];
        ou[(size_t)b * N + i] = u.x;  // ov already points at the v planes
        ov[(size_t)b * N + i] = u.y;
    }
}

void launch_upscale2(const float2 *src, size_t sstride, int w, int h, float2 *dst,
                     size_t dstride, int nw, int nh, float sx, float sy, int B,
                     cudaStream_t st) {
    dim3 blk(32, 8), g(div_up(nw, 32), div_up(nh, 8), B);
    k_upscale2<<<g, blk, 0, st>>>(src, sstride, w, h, dst, dstride, nw, nh, sx, sy);
}

// Each thread converts four consecutive pixels of a row; rows whose source and destination allow it move them as one vector.
constexpr int kTabPx = 4;
template <typename T>
__global__ void k_ingest_tab(const FrameRef *__restrict__ frames, int w, int h, float *dst,
                             size_t N) {
    const int x = (blockIdx.x * blockDim.x + threadIdx.x) * kTabPx;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const FrameRef f = frames[blockIdx.z];
    const T *src = static_cast<const T *>(f.p) + (size_t)y * f.pitch + x;
    float *d = dst + (size_t)blockIdx.z * N + (size_t)y * w + x;
    const bool vec = x + kTabPx <= w && reinterpret_cast<uintptr_t>(d) % 16 == 0 &&
                     reinterpret_cast<uintptr_t>(src) % (kTabPx * sizeof(T)) == 0;
    if (vec) {
        float4 v;
        if (sizeof(T) == 4) {
            v = __ldg(reinterpret_cast<const float4 *>(src));
        } else {
            const uchar4 c = __ldg(reinterpret_cast<const uchar4 *>(src));
            v = make_float4((float)c.x, (float)c.y, (float)c.z, (float)c.w);
        }
        *reinterpret_cast<float4 *>(d) = v;
        return;
    }
    for (int k = 0; k < kTabPx && x + k < w; k++) d[k] = (float)__ldg(src + k);
}

void launch_ingest_tab(const FrameRef *frames, int dtype, int w, int h, float *dst, size_t N,
                       int planes, cudaStream_t st) {
    dim3 blk(32, 8), g(div_up(w, 32 * kTabPx), div_up(h, 8), planes);
    if (dtype == OFLOW_U8)
        k_ingest_tab<uint8_t><<<g, blk, 0, st>>>(frames, w, h, dst, N);
    else
        k_ingest_tab<float><<<g, blk, 0, st>>>(frames, w, h, dst, N);
}

__global__ void k_split_tab(const float2 *__restrict__ U, size_t stride, int w, int h,
                            const OutRef *__restrict__ outs) {
    const int x = (blockIdx.x * blockDim.x + threadIdx.x) * kTabPx;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const OutRef o = outs[blockIdx.z];
    const float2 *s = U + (size_t)blockIdx.z * stride + (size_t)y * w + x;
    float *du = o.u + (size_t)y * o.pitch + x, *dv = o.v + (size_t)y * o.pitch + x;
    const bool vec = x + kTabPx <= w &&
                     ((reinterpret_cast<uintptr_t>(s) | reinterpret_cast<uintptr_t>(du) |
                       reinterpret_cast<uintptr_t>(dv)) % 16 == 0);
    if (vec) {
        const float4 a = reinterpret_cast<const float4 *>(s)[0];
        const float4 b = reinterpret_cast<const float4 *>(s)[1];
        *reinterpret_cast<float4 *>(du) = make_float4(a.x, a.z, b.x, b.z);
        *reinterpret_cast<float4 *>(dv) = make_float4(a.y, a.w, b.y, b.w);
        return;
    }
    for (int k = 0; k < kTabPx && x + k < w; k++) {
        const float2 u = s[k];
        du[k] = u.x;
        dv[k] = u.y;
    }
}

void launch_split_tab(const float2 *U, size_t stride, int w, int h, const OutRef *outs, int B,
                      cudaStream_t st) {
    dim3 blk(32, 8), g(div_up(w, 32 * kTabPx), div_up(h, 8), B);
    k_split_tab<<<g, blk, 0, st>>>(U, stride, w, h, outs);
}

void launch_split2(const float2 *U, size_t stride, int N, float *out, int B, cudaStream_t st) {
    k_split2<<<dim3(imin(div_up(N, 1024), 1024), B), 256, 0, st>>>(U, stride, N, out,
                                                                   out + (size_t)B * N, B);
}

// ================================================================ host plan
constexpr int kJTW = 32, kJTH = 16, kJK = 4, kJNT = 256;

// Jacobi configurations: tile tw x th, up to k sweeps per launch (halo k),
// nt threads; 36 B of shared memory per region pixel (D 16, two u buffers,
// the reciprocal of the denominator).
struct HsJCfg {
    int tw, th, k, nt;
};
constexpr HsJCfg kHsCfgs[] = {{32, 16, 4, 256}, {32, 16, 8, 256}, {64, 32, 8, 512},
                              {64, 16, 4, 256}, {32, 32, 16, 512}, {64, 32, 4, 512}};
constexpr int kHsNumCfgs = 6;
constexpr size_t hs_smem(const HsJCfg &c) { return (size_t)(c.tw + 2 * c.k) * (c.th + 2 * c.k) * 36; }

template <int TW, int TH, int KH, int NT>
static void hs_jacobi_launch(dim3 g, cudaStream_t st, const float4 *D, size_t dstride,
                             const float2 *in, float2 *out, float2 *U, size_t stride, int w,
                             int h, int sweeps, int first, int last, const HsTma &tma) {
    const size_t smem = (size_t)(TW + 2 * KH) * (TH + 2 * KH) * 36;
    k_hs_jacobi<TW, TH, KH, NT><<<g, NT, smem, st>>>(D, dstride, in, out, U, stride, w, h, sweeps,
                                                     first, last, tma);
}

static void hs_jacobi_cfg(int c, dim3 g, cudaStream_t st, const float4 *D, size_t dstride,
                          const float2 *in, float2 *out, float2 *U, size_t stride, int w, int h,
                          int sweeps, int first, int last, const HsTma &t) {
    switch (c) {
        case 1: hs_jacobi_launch<32, 16, 8, 256>(g, st, D, dstride, in, out, U, stride, w, h, sweeps, first, last, t); break;
        case 2: hs_jacobi_launch<64, 32, 8, 512>(g, st, D, dstride, in, out, U, stride, w, h, sweeps, first, last, t); break;
        case 3: hs_jacobi_launch<64, 16, 4, 256>(g, st, D, dstride, in, out, U, stride, w, h, sweeps, first, last, t); break;
        case 4: hs_jacobi_launch<32, 32, 16, 512>(g, st, D, dstride, in, out, U, stride, w, h, sweeps, first, last, t); break;
        case 5: hs_jacobi_launch<64, 32, 4, 512>(g, st, D, dstride, in, out, U, stride, w, h, sweeps, first, last, t); break;
        default: hs_jacobi_launch<32, 16, 4, 256>(g, st, D, dstride, in, out, U, stride, w, h, sweeps, first, last, t); break;
    }
}

// Tensor maps of the Jacobi region loads for configuration c on a level of
// w x h (pairs N apart, B pairs) reading increments from `in`.  TMA wants
// 16-byte strides: even w and N, else the kernel loads the region itself.
static HsTma hs_tma(int c, const float4 *D, const float2 *in, int w, int h, size_t N, int B,
                    int *err) {
    HsTma t;
    memset(&t, 0, sizeof(t));
    t.err = err;
    if ((w & 1) || (N & 1) || err == nullptr) return t;
    const HsJCfg &jc = kHsCfgs[c];
    const cuuint32_t rw = (cuuint32_t)(jc.tw + 2 * jc.k), rh = (cuuint32_t)(jc.th + 2 * jc.k);
    const cuuint64_t dd[3] = {2 * (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)B};
    const cuuint64_t sd[2] = {16 * (cuuint64_t)w, 16 * (cuuint64_t)N};
    const cuuint32_t bd[3] = {2 * rw, rh, 1};
    const cuuint64_t di[3] = {(cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)B};
    const cuuint64_t si[2] = {8 * (cuuint64_t)w, 8 * (cuuint64_t)N};
    const cuuint32_t bi[3] = {rw, rh, 1};
    t.use = encode_map8(&t.tD, const_cast<float4 *>(D), 3, dd, sd, bd) &&
            encode_map8(&t.tIn, const_cast<float2 *>(in), 3, di, si, bi);
    return t;
}

static void hs_set_smem_attrs() {
    OF_CUDA(cudaFuncSetAttribute(k_hs_jacobi<32, 16, 4, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)hs_smem(kHsCfgs[0])));
    OF_CUDA(cudaFuncSetAttribute(k_hs_jacobi<32, 16, 8, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)hs_smem(kHsCfgs[1])));
    OF_CUDA(cudaFuncSetAttribute(k_hs_jacobi<64, 32, 8, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)hs_smem(kHsCfgs[2])));
    OF_CUDA(cudaFuncSetAttribute(k_hs_jacobi<64, 16, 4, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)hs_smem(kHsCfgs[3])));
    OF_CUDA(cudaFuncSetAttribute(k_hs_jacobi<32, 32, 16, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)hs_smem(kHsCfgs[4])));
    OF_CUDA(cudaFuncSetAttribute(k_hs_jacobi<64, 32, 4, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)hs_smem(kHsCfgs[5])));
}

// OFLOW_HS_CFG forces one configuration (used to test and time them); else
// configuration 0 unless the tuning table has the level
static int hs_pick() {
    if (const char *e = getenv("OFLOW_HS_CFG")) {
        const int c = atoi(e);
        if (c >= 0 && c < kHsNumCfgs) return c;
    }
    return 0;
}

HsPlan::HsPlan(int w, int h, int B, int dtype, const oflow_hs_params &prm, const TuneTable *tuned)
    : w_(w), h_(h), B_(B), dtype_(dtype), prm_(prm) {
    OF_CHECK(B >= 1, "hs: empty batch");
    OF_CHECK(prm.nlevels >= 1 && prm.nlevels <= 16, "hs: nlevels out of range");
    OF_CHECK(prm.nwarp >= 0 && prm.nsolver >= 0, "hs: negative iteration count");
    L_ = prm.nlevels;
    W_[L_ - 1] = w;
    H_[L_ - 1] = h;
    for (int l = L_ - 1; l > 0; l--) {
        W_[l - 1] = W_[l] / 2;
        H_[l - 1] = H_[l] / 2;
    }
    OF_CHECK(W_[0] >= 1 && H_[0] >= 1, "hs: too many levels for the frame size");
    N_ = (size_t)w * h;
    size_t acc = 0;
    for (int l = 0; l < L_; l++) {
        pyr_off_[l] = acc;
        acc += (size_t)2 * B * W_[l] * H_[l];
    }
    const size_t esz = dtype == OFLOW_U8 ? 1 : 4;
    o_raw_ = ar_.reserve(2 * B * N_ * esz);
    o_pyr_ = ar_.reserve(acc * 4);
    o_D_ = ar_.reserve(B * N_ * 16);
    o_dU0_ = ar_.reserve(B * N_ * 8);
    o_dU1_ = ar_.reserve(B * N_ * 8);
    o_Ua_ = ar_.reserve(B * N_ * 8);
    o_Ub_ = ar_.reserve(B * N_ * 8);
    o_out_ = ar_.reserve(2 * B * N_ * 4);
    o_ftab_ = ar_.reserve(sizeof(FrameRef) * 2 * B);
    o_otab_ = ar_.reserve(sizeof(OutRef) * B);
    ar_.commit();
    io_.init(ar_.at<FrameRef>(o_ftab_), ar_.at<OutRef>(o_otab_), B);
    for (int b = 0; b < B; b++) {
        bind_raw(b, 0);
        bind_raw(b, 1);
        bind_own_out(b);
    }
    // the default tables are valid for schedules recorded into a caller's graph
    io_.upload(nullptr);
    OF_CUDA(cudaStreamSynchronize(nullptr));
    hs_set_smem_attrs();
    for (int l = 0; l < L_; l++) {
        const auto it = tuned ? tuned->find(tune_key(W_[l], H_[l], B, kTuneHs)) : TuneTable::const_iterator();
        const bool ok = tuned && it != tuned->end() && it->second >= 0 && it->second < kHsNumCfgs;
        jcfg_[l] = ok ? it->second : hs_pick();
    }
}

void *HsPlan::raw_input(int b, int k) const {
    const size_t esz = dtype_ == OFLOW_U8 ? 1 : 4;
    return ar_.at<char>(o_raw_) + (size_t)(2 * b + k) * N_ * esz;
}
const float *HsPlan::out_u(int b) const { return ar_.at<float>(o_out_) + (size_t)b * N_; }
const float *HsPlan::out_v(int b) const { return ar_.at<float>(o_out_) + (size_t)(B_ + b) * N_; }
void HsPlan::bind_frame(int b, int k, const void *p, int pitch) { io_.set_frame(b, k, p, pitch ? pitch : w_); }
void HsPlan::bind_raw(int b, int k) { io_.set_frame(b, k, raw_input(b, k), w_); }
void HsPlan::bind_out(int b, float *u, float *v, int pitch) { io_.set_out(b, u, v, pitch ? pitch : w_); }
void HsPlan::bind_own_out(int b) {
    float *o = ar_.at<float>(o_out_);
    io_.set_out(b, o + (size_t)b * N_, o + (size_t)(B_ + b) * N_, w_);
}

void HsPlan::record(cudaStream_t st) {
    const int B = B_;
    float *pyr = ar_.at<float>(o_pyr_);
    float4 *D = ar_.at<float4>(o_D_);
    float2 *dU[2] = {ar_.at<float2>(o_dU0_), ar_.at<float2>(o_dU1_)};
    float2 *Ubuf[2] = {ar_.at<float2>(o_Ua_), ar_.at<float2>(o_Ub_)};
    const int top = L_ - 1;
    {
        // frames through the frame table (the caller's device frames in place,
        // or this plan's staging buffers)
        launch_ingest_tab(io_.frames(), dtype_, w_, h_, pyr + pyr_off_[top], N_, 2 * B, st);
    }
    for (int l = top; l > 0; l--) {
        dim3 blk(32, 8), g(div_up(W_[l - 1], 32), div_up(H_[l - 1], 8), 2 * B);
        k_hs_downscale<<<g, blk, 0, st>>>(pyr + pyr_off_[l], (size_t)W_[l] * H_[l], W_[l], H_[l],
                                          pyr + pyr_off_[l - 1], (size_t)W_[l - 1] * H_[l - 1]);
    }
    int ub = 0;  // Ubuf index holding the flow of the current level
    OF_CUDA(cudaMemsetAsync(Ubuf[ub], 0, B * N_ * 8, st));
    for (int l = 0; l < L_; l++) {
        const HsJCfg &jc = kHsCfgs[jcfg_[l]];
        const int lw = W_[l], lh = H_[l];
        const size_t lp = (size_t)lw * lh;
        for (int wi = 0; wi < prm_.nwarp; wi++) {
            dim3 dg(div_up(lw, kDTW), div_up(lh, kDTH), B);
            k_hs_warp_deriv<<<dg, dim3(kDTW, kDTH), 0, st>>>(pyr + pyr_off_[l], lp, lw, lh,
                                                             Ubuf[ub], N_, 0, prm_.alpha, D, N_);
            dim3 jg(div_up(lw, jc.tw), div_up(lh, jc.th), B);
            int done = 0, cur = 0;
            if (prm_.nsolver == 0) continue;  // du = 0: the flow is unchanged
            while (done < prm_.nsolver) {
                const int k = imin(jc.k, prm_.nsolver - done);
                const bool first = done == 0, last = done + k == prm_.nsolver;
                const HsTma tm = hs_tma(jcfg_[l], D, dU[cur], lw, lh, N_, B, err_.device());
                hs_jacobi_cfg(jcfg_[l], jg, st, D, N_, dU[cur], dU[cur ^ 1], Ubuf[ub], N_, lw, lh, k,
                              first, last, tm);
                cur ^= 1;
                done += k;
            }
        }
        if (l != top) {
            const float sx = (float)W_[l + 1] / (float)lw;
            const float sy = (float)H_[l + 1] / (float)lh;
            launch_upscale2(Ubuf[ub], N_, lw, lh, Ubuf[ub ^ 1], N_, W_[l + 1], H_[l + 1], sx, sy, B,
                            st);
            ub ^= 1;
        }
    }
    launch_split_tab(Ubuf[ub], N_, w_, h_, io_.outs(), B, st);
    OF_CUDA(cudaGetLastError());
}

void HsPlan::run(cudaStream_t st) {
    io_.upload(st);
    if (!graph_.ready()) graph_.capture(st, [&](cudaStream_t s) { record(s); });
    graph_.launch(st);
}

// Best of `reps` timed runs of 16 sweeps (in launches of the configuration's
// depth) per configuration and level.  The sweep has no data-dependent control
// flow, so the derivative buffer the last solve left is fine input at every
// level size; the runs write only the du scratch, never the flow or outputs.
void HsPlan::autotune(cudaStream_t st, TuneTable *table, int reps) {
    float4 *D = ar_.at<float4>(o_D_);
    float2 *dU[2] = {ar_.at<float2>(o_dU0_), ar_.at<float2>(o_dU1_)};
    float2 *U = ar_.at<float2>(o_Ua_);
    cudaEvent_t e0, e1;
    OF_CUDA(cudaEventCreate(&e0));
    OF_CUDA(cudaEventCreate(&e1));
    constexpr int kSweeps = 16;
    try {
        for (int l = 0; l < L_; l++) {
            const int lw = W_[l], lh = H_[l];
            float best = 1e30f;
            int best_c = jcfg_[l];
            for (int c = 0; c < kHsNumCfgs; c++) {
                const HsJCfg &jc = kHsCfgs[c];
                dim3 jg(div_up(lw, jc.tw), div_up(lh, jc.th), B_);
                float ms_min = 1e30f;
                for (int r = 0; r <= reps; r++) {  // the first round warms up
                    OF_CUDA(cudaEventRecord(e0, st));
                    int done = 0, cur = 0;
                    while (done < kSweeps) {
                        const int k = imin(jc.k, kSweeps - done);
                        const HsTma tm = hs_tma(c, D, dU[cur], lw, lh, N_, B_, err_.device());
                        hs_jacobi_cfg(c, jg, st, D, N_, dU[cur], dU[cur ^ 1], U, N_, lw, lh, k,
                                      done == 0, 0, tm);
                        cur ^= 1;
                        done += k;
                    }
                    OF_CUDA(cudaEventRecord(e1, st));
                    OF_CUDA(cudaEventSynchronize(e1));
                    float ms = 0.0f;
                    OF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                    if (r > 0) ms_min = ms < ms_min ? ms : ms_min;
                }
                if (ms_min < best) {
                    best = ms_min;
                    best_c = c;
                }
            }
            jcfg_[l] = best_c;
            if (table) (*table)[tune_key(lw, lh, B_, kTuneHs)] = best_c;
        }
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    graph_.reset();  // the next run captures the new configurations
}

// ================================================================ caller scratch
// The Horn-Schunck schedule of HsPlan::record for one pair, enqueued on
// scratch the caller provides (no allocation here).  Frames and flows are
// device float planes with row pitches in elements.
static size_t hs_carve(size_t &off, size_t bytes) {
    const size_t at = (off + 255) & ~size_t(255);
    off = at + bytes;
    return at;
}

size_t hs_scratch_bytes(int w, int h, int nlevels) {
    if (w < 1 || h < 1 || nlevels < 1 || nlevels > 16) return 0;
    int W = w, H = h;
    size_t pyr = 0;
    for (int l = nlevels - 1; l >= 0; l--) {
        if (W < 1 || H < 1) return 0;
        pyr += (size_t)2 * W * H;
        W /= 2;
        H /= 2;
    }
    const size_t N = (size_t)w * h;
    size_t off = 0;
    hs_carve(off, pyr * 4);   // pyramid
    hs_carve(off, N * 16);    // D
    hs_carve(off, N * 8);     // dU0
    hs_carve(off, N * 8);     // dU1
    hs_carve(off, N * 8);     // Ua
    hs_carve(off, N * 8);     // Ub
    hs_carve(off, 2 * N * 4); // u | v
    return off;
}

void HsPlan::check_device_error() {
    if (err_.take()) throw Error(OFLOW_ERR_TIMEOUT, "hs: a Jacobi tile's TMA load gave up its bounded wait");
}

void hs_enqueue_into(void *scratch, const float *I0, const float *I1, int w, int h, int pitch,
                     const oflow_hs_params &prm, float *u, float *v, int out_pitch,
                     cudaStream_t st) {
    HsTma no_tma;  // this path loads its regions with plain instructions
    memset(&no_tma, 0, sizeof(no_tma));
    const int L = prm.nlevels;
    int Wl[16], Hl[16];
    Wl[L - 1] = w;
    Hl[L - 1] = h;
    for (int l = L - 1; l > 0; l--) {
        Wl[l - 1] = Wl[l] / 2;
        Hl[l - 1] = Hl[l] / 2;
    }
    size_t pyr_off[16], acc = 0;
    for (int l = 0; l < L; l++) {
        pyr_off[l] = acc;
        acc += (size_t)2 * Wl[l] * Hl[l];
    }
    const size_t N = (size_t)w * h;
    size_t off = 0;
    char *base = static_cast<char *>(scratch);
    float *pyr = reinterpret_cast<float *>(base + hs_carve(off, acc * 4));
    float4 *D = reinterpret_cast<float4 *>(base + hs_carve(off, N * 16));
    float2 *dU[2];
    dU[0] = reinterpret_cast<float2 *>(base + hs_carve(off, N * 8));
    dU[1] = reinterpret_cast<float2 *>(base + hs_carve(off, N * 8));
    float2 *Ubuf[2];
    Ubuf[0] = reinterpret_cast<float2 *>(base + hs_carve(off, N * 8));
    Ubuf[1] = reinterpret_cast<float2 *>(base + hs_carve(off, N * 8));
    float *out = reinterpret_cast<float *>(base + hs_carve(off, 2 * N * 4));
    const int top = L - 1;
    const size_t rowb = (size_t)w * 4, pb = (size_t)(pitch ? pitch : w) * 4;
    OF_CUDA(cudaMemcpy2DAsync(pyr + pyr_off[top], rowb, I0, pb, rowb, h, cudaMemcpyDeviceToDevice, st));
    OF_CUDA(cudaMemcpy2DAsync(pyr + pyr_off[top] + N, rowb, I1, pb, rowb, h,
                              cudaMemcpyDeviceToDevice, st));
    for (int l = top; l > 0; l--) {
        dim3 blk(32, 8), g(div_up(Wl[l - 1], 32), div_up(Hl[l - 1], 8), 2);
        k_hs_downscale<<<g, blk, 0, st>>>(pyr + pyr_off[l], (size_t)Wl[l] * Hl[l], Wl[l], Hl[l],
                                          pyr + pyr_off[l - 1], (size_t)Wl[l - 1] * Hl[l - 1]);
    }
    int ub = 0;
    OF_CUDA(cudaMemsetAsync(Ubuf[ub], 0, N * 8, st));  // the flow starts at zero
    const size_t smem = (size_t)(kJTW + 2 * kJK) * (kJTH + 2 * kJK) * 36;
    for (int l = 0; l < L; l++) {
        const int lw = Wl[l], lh = Hl[l];
        const size_t lp = (size_t)lw * lh;
        for (int wi = 0; wi < prm.nwarp; wi++) {
            dim3 dg(div_up(lw, kDTW), div_up(lh, kDTH), 1);
            k_hs_warp_deriv<<<dg, dim3(kDTW, kDTH), 0, st>>>(pyr + pyr_off[l], lp, lw, lh,
                                                             Ubuf[ub], N, 0, prm.alpha, D, N);
            dim3 jg(div_up(lw, kJTW), div_up(lh, kJTH), 1);
            int done = 0, cur = 0;
            while (done < prm.nsolver) {
                const int k = imin(kJK, prm.nsolver - done);
                k_hs_jacobi<kJTW, kJTH, kJK, kJNT><<<jg, kJNT, smem, st>>>(
                    D, N, dU[cur], dU[cur ^ 1], Ubuf[ub], N, lw, lh, k, done == 0,
                    done + k == prm.nsolver, no_tma);
                cur ^= 1;
                done += k;
            }
        }
        if (l != top) {
            const float sx = (float)Wl[l + 1] / (float)lw;
            const float sy = (float)Hl[l + 1] / (float)lh;
            launch_upscale2(Ubuf[ub], N, lw, lh, Ubuf[ub ^ 1], N, Wl[l + 1], Hl[l + 1], sx, sy, 1, st);
            ub ^= 1;
        }
    }
    launch_split2(Ubuf[ub], N, (int)N, out, 1, st);
    OF_CUDA(cudaGetLastError());
    const size_t ob = (size_t)(out_pitch ? out_pitch : w) * 4;
    OF_CUDA(cudaMemcpy2DAsync(u, ob, out, rowb, rowb, h, cudaMemcpyDeviceToDevice, st));
    OF_CUDA(cudaMemcpy2DAsync(v, ob, out + N, rowb, rowb, h, cudaMemcpyDeviceToDevice, st));
}

}  // namespace oflow
