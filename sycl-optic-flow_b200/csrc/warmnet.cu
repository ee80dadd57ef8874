// The warm-start network: a 4-stage encoder-decoder (32/64/96/128 channels,
// 3x3 convolutions, BF16 weights and activations, FP32 accumulation) that maps
// a frame pair to flow at 1/8 resolution.  Input: both frames box-filtered by
// 2 (so a 1024x436 pair enters at 512x218); output: flow at the size of TV-L1
// scale 3 (128x55 for 1024x436), in that scale's pixel units.
//
//   x0  [h1,w1,16]   (channels 0,1: I0/255 - 0.5, I1/255 - 0.5; 2: 4*(I1-I0)/255)
//   c1  s2 16->32   c2 32->32   c3 s2 32->64   c4 64->64
//   c5  s2 64->96   c6 96->96   c7 s2 96->128
//   up(c7) ++ c6 -> c8 224->96;  up(c8) ++ c4 -> c9 160->64;  c10 64->8 (flow in 0,1)
// ReLU after every convolution but the last.  Parameters: 606,536 weights
// plus biases, one fp32 vector (per layer: weights [K][3][3][C], then bias).
#include <cmath>
#include <cstring>
#include <vector>

#include "cnn.cuh"
#include "common.cuh"
#include "internal.hpp"
#include "warmnet.hpp"

#include <algorithm>
#include <cstdlib>

namespace oflow {

namespace {
struct LayerSpec {
    int cin, cout, stride;
    bool relu;
};
constexpr LayerSpec kLayers[10] = {{16, 32, 2, true},   {32, 32, 1, true},  {32, 64, 2, true},
                                   {64, 64, 1, true},   {64, 96, 2, true},  {96, 96, 1, true},
                                   {96, 128, 2, true},  {224, 96, 1, true}, {160, 64, 1, true},
                                   {64, 8, 1, false}};
}  // namespace

int warmnet_num_params() {
    int n = 0;
    for (const auto &L : kLayers) n += L.cout * 9 * L.cin + L.cout;
    return n;
}

WarmNet::WarmNet(int w, int h, int B) : w_(w), h_(h), B_(B) {
    OF_CHECK(B >= 1 && w >= 16 && h >= 16, "net: frames must be at least 16x16");
    hs_[1] = (h + 1) / 2;  ws_[1] = (w + 1) / 2;
    for (int k = 2; k <= 5; k++) {
        hs_[k] = (hs_[k - 1] + 1) / 2;
        ws_[k] = (ws_[k - 1] + 1) / 2;
    }
    size_t off = 0;
    for (int l = 0; l < 10; l++) {
        woff_[l] = off;
        off += (size_t)kLayers[l].cout * 9 * kLayers[l].cin;
        boff_[l] = off;
        off += kLayers[l].cout;
    }
    np_ = off;
    // activation sizes (pixels) per tensor
    const size_t p1 = (size_t)B * hs_[1] * ws_[1], p2 = (size_t)B * hs_[2] * ws_[2],
                 p3 = (size_t)B * hs_[3] * ws_[3], p4 = (size_t)B * hs_[4] * ws_[4],
                 p5 = (size_t)B * hs_[5] * ws_[5];
    const size_t act_ch[] = {16, 32, 32, 64, 64, 96, 96, 128, 224, 96, 160, 64};
    const size_t act_px[] = {p1, p2, p2, p3, p3, p4, p4, p5, p4, p4, p3, p3};
    size_t maxg = 0;
    for (int t = 0; t < 12; t++) {
        aoff_[t] = ar_.reserve(act_ch[t] * act_px[t] * 2);
        maxg = maxg > act_ch[t] * act_px[t] ? maxg : act_ch[t] * act_px[t];
        gsize_[t] = act_ch[t] * act_px[t];
        goff_[t] = ar_.reserve(act_ch[t] * act_px[t] * 4);
    }
    o_out_ = ar_.reserve(p3 * 8 * 4);
    o_gout_ = ar_.reserve(p3 * 8 * 4);
    o_p_ = ar_.reserve(np_ * 4);
    o_pb_ = ar_.reserve(np_ * 2);
    o_gp_ = ar_.reserve(np_ * 4);
    o_m_ = ar_.reserve(np_ * 4);
    o_v_ = ar_.reserve(np_ * 4);
    o_loss_ = ar_.reserve(8);
    o_err_ = ar_.reserve(sizeof(int));
    size_t bwd = 0;  // scratch of the tensor-core backward products
    for (int l = 0; l < 10; l++) bwd = std::max(bwd, conv_backward_data_umma_scratch(dims(l)));
    o_bwd_ = ar_.reserve(bwd);
    ar_.commit();
    if (const char *e = getenv("OFLOW_CNN_BWD_MMA")) bwd_mma_ = atoi(e) != 0;
    OF_CUDA(cudaMemset(ar_.at<char>(o_err_), 0, sizeof(int)));
    OF_CUDA(cudaMemset(ar_.at<char>(o_m_), 0, np_ * 4));
    OF_CUDA(cudaMemset(ar_.at<char>(o_v_), 0, np_ * 4));
    OF_CUDA(cudaMemset(ar_.at<char>(o_p_), 0, np_ * 4));
    OF_CUDA(cudaMemset(ar_.at<char>(o_pb_), 0, np_ * 2));
}

void WarmNet::set_params(const float *host, cudaStream_t st) {
    OF_CUDA(cudaMemcpyAsync(ar_.at<float>(o_p_), host, np_ * 4, cudaMemcpyHostToDevice, st));
    cnn_f32_to_bf16(ar_.at<float>(o_p_), ar_.at<__nv_bfloat16>(o_pb_), np_, st);
    OF_CUDA(cudaStreamSynchronize(st));
    step_ = 0;
    OF_CUDA(cudaMemsetAsync(ar_.at<char>(o_m_), 0, np_ * 4, st));
    OF_CUDA(cudaMemsetAsync(ar_.at<char>(o_v_), 0, np_ * 4, st));
}

void WarmNet::get_params(float *host, cudaStream_t st) const {
    OF_CUDA(cudaMemcpyAsync(host, ar_.at<float>(o_p_), np_ * 4, cudaMemcpyDeviceToHost, st));
    OF_CUDA(cudaStreamSynchronize(st));
}

ConvDims WarmNet::dims(int l) const {
    // input scale index per layer (1 = x0 resolution)
    static const int in_scale[10] = {1, 2, 2, 3, 3, 4, 4, 4, 3, 3};
    const int si = in_scale[l];
    const int so = kLayers[l].stride == 2 ? si + 1 : si;
    return ConvDims{B_, hs_[si], ws_[si], kLayers[l].cin, hs_[so], ws_[so], kLayers[l].cout,
                    kLayers[l].stride};
}

void WarmNet::forward(const void *frames, int dtype, size_t pair_stride, cudaStream_t st) {
    auto A = [&](int t) { return ar_.at<__nv_bfloat16>(aoff_[t]); };
    const __nv_bfloat16 *W = ar_.at<__nv_bfloat16>(o_pb_);
    const float *P = ar_.at<float>(o_p_);
    cnn_input(frames, dtype, w_, h_, B_, pair_stride, A(0), st);
    // tensors: 0 x0, 1 c1, 2 c2, 3 c3, 4 c4, 5 c5, 6 c6, 7 c7, 8 cat1, 9 c8, 10 cat2, 11 c9
    const int src[10] = {0, 1, 2, 3, 4, 5, 6, 8, 10, 11};
    const int dst[10] = {1, 2, 3, 4, 5, 6, 7, 9, 11, -1};
    for (int l = 0; l < 10; l++) {
        if (l == 7)
            upcat_forward(A(7), hs_[5], ws_[5], 128, A(6), hs_[4], ws_[4], 96, B_, A(8), st);
        if (l == 8)
            upcat_forward(A(9), hs_[4], ws_[4], 96, A(4), hs_[3], ws_[3], 64, B_, A(10), st);
        const ConvDims d = dims(l);
        if (l < 9)
            conv_forward(d, A(src[l]), W + woff_[l], P + boff_[l], A(dst[l]), false, kLayers[l].relu, st,
                         ar_.at<int>(o_err_));
        else
            conv_forward(d, A(src[l]), W + woff_[l], P + boff_[l], ar_.at<float>(o_out_), true, false,
                         st, ar_.at<int>(o_err_));
    }
}

double WarmNet::train_step(const void *frames, int dtype, size_t pair_stride, const float *target,
                           float lr, cudaStream_t st) {
    forward(frames, dtype, pair_stride, st);
    auto A = [&](int t) { return ar_.at<__nv_bfloat16>(aoff_[t]); };
    auto G = [&](int t) { return ar_.at<float>(goff_[t]); };
    const __nv_bfloat16 *W = ar_.at<__nv_bfloat16>(o_pb_);
    float *gp = ar_.at<float>(o_gp_);
    const int M3 = B_ * hs_[3] * ws_[3];
    flow_loss(ar_.at<float>(o_out_), 8, target, M3, ar_.at<float>(o_gout_), ar_.at<double>(o_loss_), st);
    // layer 10 (no ReLU): gradient arrives at its output
    auto back = [&](int l, const float *g, int yact_t, int x_t, float *gin, bool acc) {
        const ConvDims d = dims(l);
        const __nv_bfloat16 *yact = yact_t >= 0 ? A(yact_t) : nullptr;
        // both backward products on the tensor-core kernels where the shape
        // allows (OFLOW_CNN_BWD_MMA=1 keeps them on the mma.sync kernel, to compare)
        const bool wg = !bwd_mma_ && conv_backward_weight_umma(d, g, yact, A(x_t), gp + woff_[l],
                                                               gp + boff_[l], ar_.at<char>(o_bwd_),
                                                               ar_.at<int>(o_err_), st);
        if (!wg) conv_backward_weight(d, g, yact, A(x_t), gp + woff_[l], gp + boff_[l], st);
        // the tensor-core backward-weight product left the masked bf16
        // gradient at the start of the shared scratch
        if (gin && (bwd_mma_ || !conv_backward_data_umma(d, g, yact, W + woff_[l], gin, acc,
                                                          ar_.at<char>(o_bwd_), ar_.at<int>(o_err_), st,
                                                          wg)))
            conv_backward_data(d, g, yact, W + woff_[l], gin, acc, st);
    };
    back(9, ar_.at<float>(o_gout_), -1, 11, G(11), false);  // c10: -> g(c9)
    back(8, G(11), 11, 10, G(10), false);                   // c9 : -> g(cat2)
    OF_CUDA(cudaMemsetAsync(G(4), 0, gsize_[4] * 4, st));
    upcat_backward(G(10), hs_[3], ws_[3], 96, 64, B_, G(9), hs_[4], ws_[4], G(4), st);
    back(7, G(9), 9, 8, G(8), false);                       // c8 : -> g(cat1)
    OF_CUDA(cudaMemsetAsync(G(6), 0, gsize_[6] * 4, st));
    upcat_backward(G(8), hs_[4], ws_[4], 128, 96, B_, G(7), hs_[5], ws_[5], G(6), st);
    back(6, G(7), 7, 6, G(6), true);                        // c7 : -> g(c6) +=
    back(5, G(6), 6, 5, G(5), false);                       // c6
    back(4, G(5), 5, 4, G(4), true);                        // c5 : -> g(c4) +=
    back(3, G(4), 4, 3, G(3), false);                       // c4
    back(2, G(3), 3, 2, G(2), false);                       // c3
    back(1, G(2), 2, 1, G(1), false);                       // c2
    back(0, G(1), 1, 0, nullptr, false);                    // c1
    step_++;
    adam_step(ar_.at<float>(o_p_), gp, ar_.at<float>(o_m_), ar_.at<float>(o_v_), np_, lr, 0.9f,
              0.999f, 1e-8f, step_, st);
    cnn_f32_to_bf16(ar_.at<float>(o_p_), ar_.at<__nv_bfloat16>(o_pb_), np_, st);
    double loss = 0.0;
    OF_CUDA(cudaMemcpyAsync(&loss, ar_.at<double>(o_loss_), 8, cudaMemcpyDeviceToHost, st));
    OF_CUDA(cudaStreamSynchronize(st));
    check_device_error(st);
    return loss;
}

void WarmNet::check_device_error(cudaStream_t st) {
    int e = 0;
    OF_CUDA(cudaMemcpyAsync(&e, ar_.at<int>(o_err_), sizeof(int), cudaMemcpyDeviceToHost, st));
    OF_CUDA(cudaStreamSynchronize(st));
    if (e) {
        OF_CUDA(cudaMemsetAsync(ar_.at<int>(o_err_), 0, sizeof(int), st));
        throw Error(OFLOW_ERR_TIMEOUT, "net: a tensor-core convolution gave up a bounded wait");
    }
}

__global__ void k_flow_out(const float *out, int M, float2 *dst2, size_t stride, int pix_per_b,
                           float *dst_planar) {
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
        const float u = out[(size_t)m * 8], v = out[(size_t)m * 8 + 1];
        const int b = m / pix_per_b, p = m % pix_per_b;
        if (dst2) dst2[(size_t)b * stride + p] = make_float2(u, v);
        if (dst_planar) {
            dst_planar[(size_t)m * 2] = u;
            dst_planar[(size_t)m * 2 + 1] = v;
        }
    }
}

void WarmNet::flow_to(float2 *dst, size_t stride, float *planar, cudaStream_t st) const {
    const int P = hs_[3] * ws_[3], M = B_ * P;
    k_flow_out<<<imin(div_up(M, 256), 1024), 256, 0, st>>>(ar_.at<float>(o_out_), M, dst, stride, P,
                                                         planar);
}

}  // namespace oflow
