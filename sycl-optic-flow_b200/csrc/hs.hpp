// Batched Horn-Schunck plan (B equal-size pairs, one captured schedule).
#pragma once

#include "internal.hpp"
#include "pairio.hpp"
#include "tvl1.hpp"

namespace oflow {

class HsPlan {
  public:
    // tuned: per-level Jacobi configurations chosen by the autotuner (may be null)
    HsPlan(int w, int h, int B, int dtype, const oflow_hs_params &prm,
           const TuneTable *tuned = nullptr);
    void *raw_input(int b, int k) const;
    const float *out_u(int b) const;
    const float *out_v(int b) const;
    // Frame k of pair b: a caller's device frame (read in place on every
    // run; pitch in elements, 0 = width) or this plan's staging buffer.
    void bind_frame(int b, int k, const void *p, int pitch);
    void bind_raw(int b, int k);
    // Flow of pair b: the caller's device planes (written in place) or this
    // plan's output buffer (out_u / out_v).
    void bind_out(int b, float *u, float *v, int pitch);
    void bind_own_out(int b);
    // the frame and output tables to the device (run() does it; a caller that
    // records the schedule into its own graph does it before each launch)
    void upload_io(cudaStream_t st) { io_.upload(st); }
    void run(cudaStream_t st);
    void record(cudaStream_t st);
    // Times every Jacobi configuration (tile shape, sweeps per launch) at every
    // level on the plan's current buffers (run a solve first), keeps the
    // fastest per sweep and records it in `table`.
    void autotune(cudaStream_t st, TuneTable *table, int reps = 3);
    int levels() const { return L_; }
    int jacobi_config(int l) const { return jcfg_[l]; }
    int width() const { return w_; }
    int height() const { return h_; }
    int batch() const { return B_; }
    int dtype() const { return dtype_; }
    const oflow_hs_params &params() const { return prm_; }
    // Throws OFLOW_ERR_TIMEOUT if a Jacobi launch gave up its bounded TMA
    // wait since the last check; reads host memory only.
    void check_device_error();

  private:
    int w_, h_, B_, dtype_;
    oflow_hs_params prm_;
    int L_ = 0;
    int W_[16] = {}, H_[16] = {};
    size_t pyr_off_[16] = {};
    size_t N_ = 0;
    Arena ar_;
    size_t o_raw_ = 0, o_pyr_ = 0, o_D_ = 0, o_dU0_ = 0, o_dU1_ = 0, o_Ua_ = 0, o_Ub_ = 0,
           o_out_ = 0;
    int jcfg_[16] = {};
    Graph graph_;
    HostFlag err_;
    size_t o_ftab_ = 0, o_otab_ = 0;
    PairIo io_;
};

// Bytes of scratch hs_enqueue_into needs for one w x h pair (0: bad sizes).
size_t hs_scratch_bytes(int w, int h, int nlevels);
// One pair's Horn-Schunck schedule on caller scratch (device frames / flows).
void hs_enqueue_into(void *scratch, const float *I0, const float *I1, int w, int h, int pitch,
                     const oflow_hs_params &prm, float *u, float *v, int out_pitch,
                     cudaStream_t st);

// Shared with the pyramidal LK plan.
void launch_upscale2(const float2 *src, size_t sstride, int w, int h, float2 *dst,
                     size_t dstride, int nw, int nh, float sx, float sy, int B, cudaStream_t st);
void launch_split2(const float2 *U, size_t stride, int N, float *out, int B, cudaStream_t st);

}  // namespace oflow
