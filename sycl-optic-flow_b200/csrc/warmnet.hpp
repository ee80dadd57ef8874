// The warm-start network (fixed architecture; see warmnet.cu).
#pragma once

#include "cnn.cuh"
#include "internal.hpp"

namespace oflow {

int warmnet_num_params();

class WarmNet {
  public:
    // w, h: full-resolution frame size; B: pairs per call
    WarmNet(int w, int h, int B);
    int width() const { return w_; }
    int height() const { return h_; }
    int batch() const { return B_; }
    // output flow size (TV-L1 scale 3 of a w x h frame)
    int out_w() const { return ws_[3]; }
    int out_h() const { return hs_[3]; }
    size_t num_params() const { return np_; }
    void set_params(const float *host, cudaStream_t st);
    void get_params(float *host, cudaStream_t st) const;
    // frames: device planes, pair b frame k at frames + (2b+k)*pair_stride
    // elements, dense w x h, dtype OFLOW_U8 / OFLOW_F32
    void forward(const void *frames, int dtype, size_t pair_stride, cudaStream_t st);
    // forward, Charbonnier loss against target f32 [B][out_h][out_w][2],
    // backward and one Adam step; returns the mean loss
    double train_step(const void *frames, int dtype, size_t pair_stride, const float *target,
                      float lr, cudaStream_t st);
    // last forward's flow into dst[b*stride + p] (float2) and/or planar
    // [B][out_h][out_w][2] floats
    void flow_to(float2 *dst, size_t stride, float *planar, cudaStream_t st) const;
    // throws OFLOW_ERR_TIMEOUT if a tensor-core convolution gave up a bounded
    // wait since the last check (synchronises st), and clears the flag
    void check_device_error(cudaStream_t st);

  private:
    ConvDims dims(int l) const;
    int w_, h_, B_;
    int hs_[6] = {}, ws_[6] = {};
    size_t woff_[10] = {}, boff_[10] = {};
    size_t np_ = 0;
    Arena ar_;
    size_t aoff_[12] = {}, goff_[12] = {}, gsize_[12] = {};
    size_t o_out_ = 0, o_gout_ = 0, o_p_ = 0, o_pb_ = 0, o_gp_ = 0, o_m_ = 0, o_v_ = 0,
           o_loss_ = 0, o_err_ = 0, o_bwd_ = 0;
    bool bwd_mma_ = false;  // backward products on the mma.sync kernel only
    int step_ = 0;
};

}  // namespace oflow
