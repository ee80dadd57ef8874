// Lucas-Kanade plans: the reference's single step over a device frame ring,
// and the pyramidal, iterated variant (B equal-size pairs).
#pragma once

#include "internal.hpp"
#include "pairio.hpp"
#include "tvl1.hpp"

namespace oflow {

int lk_taps(int spac, int temp, float *fs, float *ft);

class LkPlan {
  public:
    LkPlan(int w, int h, const oflow_lk_params &prm);
    uint8_t *ring_slot(int k) const;  // dense w*h uint8 plane of ring slot k
    const float *out_u() const;
    const float *out_v() const;
    void run(int iframe, cudaStream_t st);
    int width() const { return w_; }
    int height() const { return h_; }
    const oflow_lk_params &params() const { return prm_; }

  private:
    int w_, h_;
    oflow_lk_params prm_;
    size_t N_ = 0;
    Arena ar_;
    size_t o_ring_ = 0, o_out_ = 0;
};

class PyrLkPlan {
  public:
    PyrLkPlan(int w, int h, int B, int dtype, const oflow_lk_params &prm);
    void *raw_input(int b, int k) const;
    const float *out_u(int b) const;
    const float *out_v(int b) const;
    // frame / flow bindings as in HsPlan (caller's device buffers in place,
    // or this plan's staging and output buffers)
    void bind_frame(int b, int k, const void *p, int pitch);
    void bind_raw(int b, int k);
    void bind_out(int b, float *u, float *v, int pitch);
    void bind_own_out(int b);
    void run(cudaStream_t st);
    void record(cudaStream_t st);
    int width() const { return w_; }
    int height() const { return h_; }
    int batch() const { return B_; }
    int dtype() const { return dtype_; }
    const oflow_lk_params &params() const { return prm_; }

  private:
    int w_, h_, B_, dtype_;
    oflow_lk_params prm_;
    GaussTaps taps_{};
    int L_ = 0;
    int W_[16] = {}, H_[16] = {};
    size_t pyr_off_[16] = {};
    size_t N_ = 0;
    Arena ar_;
    size_t o_raw_ = 0, o_T_ = 0, o_pyr_ = 0, o_G_ = 0, o_U0_ = 0, o_U1_ = 0, o_out_ = 0;
    size_t o_ftab_ = 0, o_otab_ = 0;
    PairIo io_;
    Graph graph_;
};

}  // namespace oflow
