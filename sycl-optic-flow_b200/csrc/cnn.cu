// BF16 tensor-core implicit-GEMM convolutions and element-wise kernels of the
// warm-start network (see cnn.cuh for the products and layouts).
#include "cnn.cuh"
#include "common.cuh"
#include "internal.hpp"

namespace oflow {

constexpr int kCBM = 64, kCBN = 64, kCBK = 16, kCNT = 128;
constexpr int kSplitK = 2048;  // pixels per block in the weight gradient

__device__ __forceinline__ uint32_t ld_pair(const __nv_bfloat16 *p) {
    return *reinterpret_cast<const uint32_t *>(p);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Masked output gradient element (ReLU after the layer when y_act != null).
__device__ __forceinline__ float grad_at(const float *g, const __nv_bfloat16 *y_act, size_t i) {
    const float v = g[i];
    if (y_act && !(__bfloat162float(y_act[i]) > 0.0f)) return 0.0f;
    return v;
}

template <int MODE>
__global__ void __launch_bounds__(kCNT) k_conv_gemm(ConvDims d, const void *a_src,
                                                    const __nv_bfloat16 *y_act,
                                                    const __nv_bfloat16 *b_src, void *out,
                                                    const float *bias, int flags) {
    // GEMM shape of this product
    int M, NC, KD;
    if (MODE == kConvFwd) {
        M = d.N * d.P * d.Q; NC = d.K; KD = 9 * d.C;
    } else if (MODE == kConvBwdData) {
        M = d.N * d.H * d.W; NC = d.C; KD = 9 * d.K;
    } else {
        M = d.K; NC = 9 * d.C; KD = d.N * d.P * d.Q;
    }
    const int m0 = blockIdx.x * kCBM, n0 = blockIdx.y * kCBN;
    int kbeg = 0, kend = KD;
    if (MODE == kConvBwdWeight) {
        kbeg = blockIdx.z * kSplitK;
        kend = imin(KD, kbeg + kSplitK);
    }
    __shared__ __align__(16) __nv_bfloat16 As[kCBM][kCBK + 8];
    __shared__ __align__(16) __nv_bfloat16 Bs[kCBN][kCBK + 8];  // [n][k]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gid = lane >> 2, tq = lane & 3;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[i][j][e] = 0.0f;

    for (int kb = kbeg; kb < kend; kb += kCBK) {
        for (int e = tid; e < kCBM * kCBK; e += kCNT) {
            const int mm = e / kCBK, kk = e % kCBK;
            const int m = m0 + mm, k = kb + kk;
            float v = 0.0f;
            if (m < M && k < kend) {
                if (MODE == kConvFwd) {
                    const int q = m % d.Q, t = m / d.Q, p = t % d.P, n = t / d.P;
                    const int tap = k / d.C, c = k % d.C;
                    const int y = p * d.stride + tap / 3 - 1, x = q * d.stride + tap % 3 - 1;
                    if (y >= 0 && y < d.H && x >= 0 && x < d.W)
                        v = __bfloat162float(static_cast<const __nv_bfloat16 *>(a_src)[
                            (((size_t)n * d.H + y) * d.W + x) * d.C + c]);
                } else if (MODE == kConvBwdData) {
                    const int x = m % d.W, t = m / d.W, y = t % d.H, n = t / d.H;
                    const int tap = k / d.K, kc = k % d.K;
                    const int py = y + 1 - tap / 3, qx = x + 1 - tap % 3;
                    if (py >= 0 && qx >= 0 && (d.stride == 1 || ((py & 1) == 0 && (qx & 1) == 0))) {
                        const int p = py / d.stride, q = qx / d.stride;
                        if (p < d.P && q < d.Q)
                            v = grad_at(static_cast<const float *>(a_src), y_act,
                                        (((size_t)n * d.P + p) * d.Q + q) * d.K + kc);
                    }
                } else {
                    v = grad_at(static_cast<const float *>(a_src), y_act, (size_t)k * d.K + m);
                }
            }
            As[mm][kk] = __float2bfloat16(v);
        }
        for (int e = tid; e < kCBN * kCBK; e += kCNT) {
            const int nn = e / kCBK, kk = e % kCBK;
            const int col = n0 + nn, k = kb + kk;
            __nv_bfloat16 v = __float2bfloat16(0.0f);
            if (col < NC && k < kend) {
                if (MODE == kConvFwd) {
                    const int tap = k / d.C, c = k % d.C;
                    v = b_src[((size_t)col * 9 + tap) * d.C + c];
                } else if (MODE == kConvBwdData) {
                    const int tap = k / d.K, kc = k % d.K;
                    v = b_src[((size_t)kc * 9 + tap) * d.C + col];
                } else {
                    const int q = k % d.Q, t = k / d.Q, p = t % d.P, n = t / d.P;
                    const int tap = col / d.C, c = col % d.C;
                    const int y = p * d.stride + tap / 3 - 1, x = q * d.stride + tap % 3 - 1;
                    if (y >= 0 && y < d.H && x >= 0 && x < d.W)
                        v = b_src[(((size_t)n * d.H + y) * d.W + x) * d.C + c];
                }
            }
            Bs[nn][kk] = v;
        }
        __syncthreads();
        uint32_t a[2][4], b[4][2];
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const int r = wm + i * 16 + gid;
            a[i][0] = ld_pair(&As[r][tq * 2]);
            a[i][1] = ld_pair(&As[r + 8][tq * 2]);
            a[i][2] = ld_pair(&As[r][tq * 2 + 8]);
            a[i][3] = ld_pair(&As[r + 8][tq * 2 + 8]);
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int nn = wn + j * 8 + gid;
            b[j][0] = ld_pair(&Bs[nn][tq * 2]);
            b[j][1] = ld_pair(&Bs[nn][tq * 2 + 8]);
        }
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
            for (int j = 0; j < 4; j++)
                mma_bf16(acc[i][j], a[i][0], a[i][1], a[i][2], a[i][3], b[j][0], b[j][1]);
        __syncthreads();
    }
    // epilogue
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int row = m0 + wm + i * 16 + gid + (e >= 2 ? 8 : 0);
                const int col = n0 + wn + j * 8 + tq * 2 + (e & 1);
                if (row >= M || col >= NC) continue;
                float v = acc[i][j][e];
                if (MODE == kConvFwd) {
                    v += bias[col];
                    if (flags & 1) v = fmaxf(v, 0.0f);
                    if (flags & 2)
                        static_cast<float *>(out)[(size_t)row * NC + col] = v;
                    else
                        static_cast<__nv_bfloat16 *>(out)[(size_t)row * NC + col] = __float2bfloat16(v);
                } else if (MODE == kConvBwdData) {
                    float *o = static_cast<float *>(out) + (size_t)row * NC + col;
                    *o = (flags & 4) ? *o + v : v;
                } else {
                    atomicAdd(static_cast<float *>(out) + (size_t)row * NC + col, v);
                }
            }
}

// bias gradient: gb[k] = sum over pixels of the masked output gradient
__global__ void k_bias_grad(const float *g, const __nv_bfloat16 *y_act, int M, int K, float *gb) {
    const int k = blockIdx.x;
    float s = 0.0f;
    for (int m = threadIdx.x; m < M; m += blockDim.x) s += grad_at(g, y_act, (size_t)m * K + k);
    __shared__ float sh[256];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) gb[k] = sh[0];
}

void conv_forward(const ConvDims &d, const __nv_bfloat16 *x, const __nv_bfloat16 *w,
                  const float *bias, void *y, bool y_f32, bool relu, cudaStream_t st, int *err) {
    if (err && conv_forward_umma(d, x, w, bias, y, y_f32, relu, err, st)) return;
    const int M = d.N * d.P * d.Q;
    dim3 g(div_up(M, kCBM), div_up(d.K, kCBN));
    k_conv_gemm<kConvFwd><<<g, kCNT, 0, st>>>(d, x, nullptr, w, y, bias,
                                              (relu ? 1 : 0) | (y_f32 ? 2 : 0));
}

void conv_backward_data(const ConvDims &d, const float *g, const __nv_bfloat16 *y_act,
                        const __nv_bfloat16 *w, float *gin, bool accumulate, cudaStream_t st) {
    const int M = d.N * d.H * d.W;
    dim3 gr(div_up(M, kCBM), div_up(d.C, kCBN));
    k_conv_gemm<kConvBwdData><<<gr, kCNT, 0, st>>>(d, g, y_act, w, gin, nullptr,
                                                   accumulate ? 4 : 0);
}

void conv_bias_grad(const ConvDims &d, const float *g, const __nv_bfloat16 *y_act, float *gb,
                    cudaStream_t st) {
    k_bias_grad<<<d.K, 256, 0, st>>>(g, y_act, d.N * d.P * d.Q, d.K, gb);
}

void conv_backward_weight(const ConvDims &d, const float *g, const __nv_bfloat16 *y_act,
                          const __nv_bfloat16 *x, float *gw, float *gb, cudaStream_t st) {
    const int KD = d.N * d.P * d.Q;
    OF_CUDA(cudaMemsetAsync(gw, 0, sizeof(float) * (size_t)d.K * 9 * d.C, st));
    dim3 gr(div_up(d.K, kCBM), div_up(9 * d.C, kCBN), div_up(KD, kSplitK));
    k_conv_gemm<kConvBwdWeight><<<gr, kCNT, 0, st>>>(d, g, y_act, x, gw, nullptr, 0);
    k_bias_grad<<<d.K, 256, 0, st>>>(g, y_act, KD, d.K, gb);
}

__global__ void k_f32_to_bf16(const float *s, __nv_bfloat16 *d, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        d[i] = __float2bfloat16(s[i]);
}

void cnn_f32_to_bf16(const float *src, __nv_bfloat16 *dst, size_t n, cudaStream_t st) {
    k_f32_to_bf16<<<imin((int)((n + 255) / 256), 4096), 256, 0, st>>>(src, dst, n);
}

__global__ void k_upcat(const __nv_bfloat16 *lo, int Hl, int Wl, int Ca, const __nv_bfloat16 *skip,
                        int H, int W, int Cb, int N, __nv_bfloat16 *out) {
    const int C = Ca + Cb;
    const size_t total = (size_t)N * H * W * C;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const size_t pix = i / C;
        const int x = (int)(pix % W), y = (int)((pix / W) % H), n = (int)(pix / ((size_t)W * H));
        out[i] = c < Ca ? lo[(((size_t)n * Hl + imin(y / 2, Hl - 1)) * Wl + imin(x / 2, Wl - 1)) * Ca + c]
                        : skip[pix * Cb + (c - Ca)];
    }
}

// The same copy in 16-byte chunks (8 channels) when both channel counts are
// multiples of 8: one output row (n, y) per block step.
__global__ void k_upcat_v(const uint4 *lo, int Hl, int Wl, int Ca8, const uint4 *skip, int H, int W,
                          int Cb8, int N, uint4 *out) {
    const int C8 = Ca8 + Cb8, per_row = W * C8;
    for (int row = blockIdx.x; row < N * H; row += gridDim.x) {
        const int n = row / H, y = row - n * H;
        const uint4 *lrow = lo + ((size_t)n * Hl + imin(y / 2, Hl - 1)) * Wl * Ca8;
        const uint4 *srow = skip + (size_t)row * W * Cb8;
        uint4 *orow = out + (size_t)row * per_row;
        for (int e = threadIdx.x; e < per_row; e += blockDim.x) {
            const int x = e / C8, c = e - x * C8;
            orow[e] = c < Ca8 ? lrow[imin(x / 2, Wl - 1) * Ca8 + c] : srow[x * Cb8 + c - Ca8];
        }
    }
}

void upcat_forward(const __nv_bfloat16 *lo, int Hl, int Wl, int Ca, const __nv_bfloat16 *skip,
                   int H, int W, int Cb, int N, __nv_bfloat16 *out, cudaStream_t st) {
    const auto a16 = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
    if (Ca % 8 == 0 && Cb % 8 == 0 && a16(lo) && a16(skip) && a16(out)) {
        const int nb = imin(N * H, 8 * kNumSMs);
        if (nb > 0)
            k_upcat_v<<<nb, 256, 0, st>>>(reinterpret_cast<const uint4 *>(lo), Hl, Wl, Ca / 8,
                                          reinterpret_cast<const uint4 *>(skip), H, W, Cb / 8, N,
                                          reinterpret_cast<uint4 *>(out));
        return;
    }
    const size_t total = (size_t)N * H * W * (Ca + Cb);
    k_upcat<<<imin((int)((total + 255) / 256), 8192), 256, 0, st>>>(lo, Hl, Wl, Ca, skip, H, W, Cb,
                                                                    N, out);
}

// glo[n][Y][X][c] = sum of g over the children (y, x) with y/2 = Y, x/2 = X
// (children clamped into the low-resolution grid as in the forward pass)
__global__ void k_upcat_bwd_lo(const float *g, int H, int W, int Ca, int Cb, int N, float *glo,
                               int Hl, int Wl) {
    const int C = Ca + Cb;
    const size_t total = (size_t)N * Hl * Wl * Ca;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % Ca);
        const size_t pix = i / Ca;
        const int X = (int)(pix % Wl), Y = (int)((pix / Wl) % Hl), n = (int)(pix / ((size_t)Wl * Hl));
        float s = 0.0f;
        const int y1 = (Y == Hl - 1) ? H - 1 : imin(2 * Y + 1, H - 1);
        const int x1 = (X == Wl - 1) ? W - 1 : imin(2 * X + 1, W - 1);
        for (int y = 2 * Y; y <= y1; y++)
            for (int x = 2 * X; x <= x1; x++) s += g[(((size_t)n * H + y) * W + x) * C + c];
        glo[i] = s;
    }
}

__global__ void k_upcat_bwd_skip(const float *g, int H, int W, int Ca, int Cb, int N, float *gskip) {
    const int C = Ca + Cb;
    const size_t total = (size_t)N * H * W * Cb;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % Cb);
        const size_t pix = i / Cb;
        gskip[i] += g[pix * C + Ca + c];
    }
}

void upcat_backward(const float *g, int H, int W, int Ca, int Cb, int N, float *glo, int Hl,
                    int Wl, float *gskip, cudaStream_t st) {
    const size_t tl = (size_t)N * Hl * Wl * Ca, ts = (size_t)N * H * W * Cb;
    k_upcat_bwd_lo<<<imin((int)((tl + 255) / 256), 8192), 256, 0, st>>>(g, H, W, Ca, Cb, N, glo, Hl, Wl);
    k_upcat_bwd_skip<<<imin((int)((ts + 255) / 256), 8192), 256, 0, st>>>(g, H, W, Ca, Cb, N, gskip);
}

template <typename T>
__global__ void k_cnn_input(const T *frames, int w, int h, int N, size_t pair_stride,
                            __nv_bfloat16 *x0) {
    // one output row (pair n, half-resolution row y) per block step; a
    // pixel's 16 channels (32 bytes) leave as two 16-byte stores
    const int w2 = (w + 1) / 2, h2 = (h + 1) / 2;
    const int rows = N * h2;
    for (int row = blockIdx.x; row < rows; row += gridDim.x) {
        const int n = row / h2, y = row - n * h2;
        const int ya = 2 * y, yb = imin(2 * y + 1, h - 1);
        const T *f0 = frames + pair_stride * (2 * (size_t)n);
        const T *f1 = frames + pair_stride * (2 * (size_t)n + 1);
        for (int x = threadIdx.x; x < w2; x += blockDim.x) {
            const int xa = 2 * x, xb = imin(2 * x + 1, w - 1);
            float m[2];
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const T *f = k ? f1 : f0;
                const float s = (float)f[(size_t)ya * w + xa] + (float)f[(size_t)ya * w + xb] +
                                (float)f[(size_t)yb * w + xa] + (float)f[(size_t)yb * w + xb];
                m[k] = s * (0.25f / 255.0f);
            }
            const __nv_bfloat162 c01 = __floats2bfloat162_rn(m[0] - 0.5f, m[1] - 0.5f);
            const __nv_bfloat162 c23 = __floats2bfloat162_rn(4.0f * (m[1] - m[0]), 0.0f);
            uint4 lo;
            lo.x = *reinterpret_cast<const uint32_t *>(&c01);
            lo.y = *reinterpret_cast<const uint32_t *>(&c23);
            lo.z = 0u;
            lo.w = 0u;
            uint4 *o = reinterpret_cast<uint4 *>(x0 + ((size_t)row * w2 + x) * 16);
            o[0] = lo;
            o[1] = make_uint4(0u, 0u, 0u, 0u);
        }
    }
}

void cnn_input(const void *frames, int dtype, int w, int h, int N, size_t pair_stride,
               __nv_bfloat16 *x0, cudaStream_t st) {
    const int nb = imin(N * ((h + 1) / 2), 8 * kNumSMs);
    if (nb <= 0) return;
    OF_CHECK((reinterpret_cast<uintptr_t>(x0) & 15u) == 0, "cnn_input: x0 not 16-byte aligned");
    if (dtype == OFLOW_U8)
        k_cnn_input<uint8_t><<<nb, 256, 0, st>>>(static_cast<const uint8_t *>(frames), w, h, N,
                                                 pair_stride, x0);
    else
        k_cnn_input<float><<<nb, 256, 0, st>>>(static_cast<const float *>(frames), w, h, N,
                                               pair_stride, x0);
}

__global__ void k_flow_loss(const float *pred, int Kp, const float *tgt, int M, float *g,
                            double *loss) {
    __shared__ double sh[256];
    double s = 0.0;
    const float eps2 = 1e-6f;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
        for (int c = 0; c < Kp; c++) {
            float gv = 0.0f;
            if (c < 2) {
                const float dlt = pred[(size_t)m * Kp + c] - tgt[(size_t)m * 2 + c];
                const float r = sqrtf(dlt * dlt + eps2);
                s += (double)r;
                gv = dlt / r / (float)(2 * M);
            }
            g[(size_t)m * Kp + c] = gv;
        }
    }
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, sh[0] / (double)(2 * M));
}

void flow_loss(const float *pred, int Kp, const float *target, int M, float *g, double *loss,
               cudaStream_t st) {
    OF_CUDA(cudaMemsetAsync(loss, 0, sizeof(double), st));
    k_flow_loss<<<imin(div_up(M, 256), 1024), 256, 0, st>>>(pred, Kp, target, M, g, loss);
}

__global__ void k_adam(float *p, const float *gp, float *m, float *v, size_t n, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float g = gp[i];
        const float mi = b1 * m[i] + (1.0f - b1) * g;
        const float vi = b2 * v[i] + (1.0f - b2) * g * g;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

void adam_step(float *p, const float *gp, float *m, float *v, size_t n, float lr, float b1,
               float b2, float eps, int t, cudaStream_t st) {
    const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
    k_adam<<<imin((int)((n + 255) / 256), 4096), 256, 0, st>>>(p, gp, m, v, n, lr, b1, b2, eps, c1, c2);
}

}  // namespace oflow
