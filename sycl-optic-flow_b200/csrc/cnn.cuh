// BF16 tensor-core convolution kernels (3x3, pad 1, stride 1 or 2) written as
// implicit GEMMs with FP32 accumulation, and the small element-wise kernels
// the warm-start network needs.  Layout: activations NHWC, weights [K][3][3][C]
// (output channel, tap row, tap column, input channel).
//
// One generic kernel covers the three products of a convolution layer:
//   forward      out[m=(n,p,q)][k]      = sum_{r,s,c} x[n][p*st+r-1][q*st+s-1][c] w[k][r][s][c]
//   backward-in  gin[m=(n,y,x)][c]      = sum_{r,s,k} g[n][(y+1-r)/st][(x+1-s)/st][k] w[k][r][s][c]
//                                         (taps whose division is inexact or out of range are 0)
//   backward-w   gw[k][(r,s,c)]        += sum_{n,p,q} g[n][p][q][k] x[n][p*st+r-1][q*st+s-1][c]
// Operands are gathered into shared memory tile by tile (BM x 16 and 16 x BN
// bf16), multiplied with mma.sync.m16n8k16 (bf16 in, f32 accumulate).  With a
// ReLU after the layer, the output gradient is masked by (out > 0) while it is
// gathered.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace oflow {

enum ConvMode { kConvFwd = 0, kConvBwdData = 1, kConvBwdWeight = 2 };

struct ConvDims {
    int N, H, W, C;   // input activations
    int P, Q, K;      // output activations
    int stride;
};

inline int conv_out(int n, int stride) { return stride == 1 ? n : (n + 1) / 2; }

// forward: x bf16 [N,H,W,C], w bf16 [K,3,3,C], bias f32 [K] -> y [N,P,Q,K]
// (bf16, or f32 when y_f32); relu applies max(0, .).  With err (a device int)
// the tcgen05 kernel runs where the shape allows (C % 16 == 0, K <= 128) and
// sets *err if one of its bounded waits gave up; otherwise, and without err,
// the mma.sync kernel runs.
void conv_forward(const ConvDims &d, const __nv_bfloat16 *x, const __nv_bfloat16 *w,
                  const float *bias, void *y, bool y_f32, bool relu, cudaStream_t st,
                  int *err = nullptr);
// the tcgen05 form alone; false (nothing launched) when the shape is outside it.
// ldy: elements between output rows (0: K); accumulate: y += (f32 output
// only); bias may be null.  A negative d.stride (-2) reads the input dilated
// by 2, the gather of a stride-2 layer's backward-data product.
bool conv_forward_umma(const ConvDims &d, const __nv_bfloat16 *x, const __nv_bfloat16 *w,
                       const float *bias, void *y, bool y_f32, bool relu, int *err, cudaStream_t st,
                       int ldy = 0, bool accumulate = false);
// backward-data on the tcgen05 kernel: the ReLU-masked gradient rounded to
// bf16 and the rotated, transposed weights go to `scratch`
// (conv_backward_data_umma_scratch bytes), then the product runs as forward
// convolutions of at most 128 output channels each; a K that is not a
// multiple of 16 is padded to one (zero channels, zero weights).  false
// (nothing launched) when K is not a multiple of 8, C not one of 16, or gin is
// not 16-byte aligned.
size_t conv_backward_data_umma_scratch(const ConvDims &d);
// backward-weight on the tcgen05 kernel (MN-major operands gathered from NHWC
// memory, reduction over output pixels split across CTAs, atomics into gw);
// gw and gb are overwritten; for K % 4 == 0 the bias gradient is a fixed-order
// sum of per-block partial sums made in the pass that masks the gradient.
// scratch: the same size as for backward-data.  false (nothing launched) when
// K > 128, K is not a multiple of 8, C not one of 16, or x or scratch is not
// 16-byte aligned.
bool conv_backward_weight_umma(const ConvDims &d, const float *g, const __nv_bfloat16 *y_act,
                               const __nv_bfloat16 *x, float *gw, float *gb, void *scratch,
                               int *err, cudaStream_t st);
// bias gradient alone: gb[k] = sum over output pixels of the masked gradient
void conv_bias_grad(const ConvDims &d, const float *g, const __nv_bfloat16 *y_act, float *gb,
                    cudaStream_t st);
// g_masked: scratch already holds the masked bf16 gradient (the backward-weight
// product on the same scratch and gradient wrote it), so it is not made again.
bool conv_backward_data_umma(const ConvDims &d, const float *g, const __nv_bfloat16 *y_act,
                             const __nv_bfloat16 *w, float *gin, bool accumulate, void *scratch,
                             int *err, cudaStream_t st, bool g_masked = false);
// backward-data: g f32 [N,P,Q,K] (masked by y_act > 0 when y_act != null,
// y_act bf16 [N,P,Q,K]) -> gin f32 [N,H,W,C]; accumulate adds to gin.
void conv_backward_data(const ConvDims &d, const float *g, const __nv_bfloat16 *y_act,
                        const __nv_bfloat16 *w, float *gin, bool accumulate, cudaStream_t st);
// backward-weight: gw f32 [K,3,3,C] and gb f32 [K] are overwritten.
void conv_backward_weight(const ConvDims &d, const float *g, const __nv_bfloat16 *y_act,
                          const __nv_bfloat16 *x, float *gw, float *gb, cudaStream_t st);

// element-wise helpers
void cnn_f32_to_bf16(const float *src, __nv_bfloat16 *dst, size_t n, cudaStream_t st);
// out[n][y][x][0..Ca) = lo[n][y/2][x/2][:], out[...][Ca..Ca+Cb) = skip[n][y][x][:]
void upcat_forward(const __nv_bfloat16 *lo, int Hl, int Wl, int Ca, const __nv_bfloat16 *skip,
                   int H, int W, int Cb, int N, __nv_bfloat16 *out, cudaStream_t st);
// gradient of upcat: glo (overwritten) and gskip (added to)
void upcat_backward(const float *g, int H, int W, int Ca, int Cb, int N, float *glo, int Hl,
                    int Wl, float *gskip, cudaStream_t st);
// network input: 2x2 box of two frames (u8 or f32, dense w x h, pair stride),
// scaled to [0,1]: channel 0 = I0 - 0.5, 1 = I1 - 0.5, 2 = 4*(I1 - I0), the
// rest 0, of a [N, ceil(h/2), ceil(w/2), 16] bf16 tensor
void cnn_input(const void *frames, int dtype, int w, int h, int N, size_t pair_stride,
               __nv_bfloat16 *x0, cudaStream_t st);
// Charbonnier loss between flow channels (0,1) of pred f32 [M,Kp] and target
// f32 [M,2]; writes the gradient into g f32 [M,Kp] (other channels 0) and the
// loss sum into loss (one double).
void flow_loss(const float *pred, int Kp, const float *target, int M, float *g, double *loss,
               cudaStream_t st);
// Adam on fp32 parameters, then bf16 copies of the weights.
void adam_step(float *p, const float *gp, float *m, float *v, size_t n, float lr, float b1,
               float b2, float eps, int t, cudaStream_t st);

}  // namespace oflow
