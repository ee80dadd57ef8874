// Drop-in C++ shims with the reference's solver entry points, implemented over
// the C ABI of oflow.h (header-only; link liboflow.so).
//
//   TV_L1                  src/tvl1/sequential/tvl1.hpp:10-17 (uint8 pair) and
//                          src/tvl1/cuda/tvl1.cuh:12-20 (streaming float frames)
//   initFlow / ComputeFlow / deleteFlow_mem
//                          src/hs/cuda/flow.cuh:19-33
//   LucasKanade            src/lk/cuda/lucaskanade.cuh:6-12
//
// Same names, argument meaning and output layout.  Errors throw
// oflow::compat_error (the reference terminates or exits instead); the
// status code and the context's message are kept in the exception.
#ifndef OFLOW_COMPAT_HPP
#define OFLOW_COMPAT_HPP

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "oflow.h"

namespace oflow {

struct compat_error : std::runtime_error {
    oflow_status status;
    compat_error(oflow_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

inline void compat_check(oflow_status s, const oflow_ctx *ctx) {
    if (s != OFLOW_OK)
        throw compat_error(s, std::string(oflow_status_string(s)) +
                                  (ctx ? std::string(": ") + oflow_ctx_last_error(ctx) : ""));
}

// One context per process for the free-function HS interface (the reference
// keeps its HS state in globals too, src/hs/cuda/flow.cu:26-44).
inline oflow_ctx *&compat_global_ctx() {
    static oflow_ctx *ctx = nullptr;
    return ctx;
}

}  // namespace oflow

// ------------------------------------------------------------------ TV-L1
class TV_L1 {
  public:
    TV_L1(int width, int height, float tau = 0.25, float lambda = 0.15, float theta = 0.3,
          int nscales = 100, float zfactor = 0.5, int warps = 5, float epsilon = 0.01,
          int max_iterations = 300, int device = 0)
        : w_(width), h_(height), u_(2 * (size_t)width * height, 0.0f) {
        p_.tau = tau;
        p_.lambda = lambda;
        p_.theta = theta;
        p_.nscales = nscales;
        p_.zfactor = zfactor;
        p_.warps = warps;
        p_.epsilon = epsilon;
        p_.max_iterations = max_iterations;
        oflow::compat_check(oflow_ctx_create(device, &ctx_), nullptr);
    }
    ~TV_L1() {
        if (stream_) oflow_stream_destroy(stream_);
        oflow_ctx_destroy(ctx_);
    }
    TV_L1(const TV_L1 &) = delete;
    TV_L1 &operator=(const TV_L1 &) = delete;

    // Sequential form: two uint8 frames (tvl1.hpp:17).
    void runDualTVL1Multiscale(uint8_t *I0, uint8_t *I1) {
        const oflow_image a{I0, w_, h_, 0, OFLOW_U8, OFLOW_HOST};
        const oflow_image b{I1, w_, h_, 0, OFLOW_U8, OFLOW_HOST};
        solve(a, b);
    }
    // Streaming form: one float frame, paired with the previous call's frame
    // (tvl1.cuh:19, tvl1.cu:122-130); before the first frame it is all zeros.
    // The previous frame stays on the device (oflow_stream): one upload per call.
    void runDualTVL1Multiscale(const float *I) {
        if (!stream_) {
            oflow_stream_desc d{};
            d.solver = OFLOW_SOLVER_TVL1;
            d.width = w_;
            d.height = h_;
            d.dtype = OFLOW_F32;
            d.lanes = 1;
            d.tvl1 = p_;
            oflow::compat_check(oflow_stream_create(ctx_, &d, &stream_), ctx_);
        }
        const oflow_image f{I, w_, h_, 0, OFLOW_F32, OFLOW_HOST};
        const oflow_flow o{u_.data(), u_.data() + (size_t)w_ * h_, 0, OFLOW_HOST};
        oflow::compat_check(oflow_stream_push(stream_, &f, &o, &st_), ctx_);
    }
    // Planar [u (w*h) | v (w*h)], valid until the next call.
    float *getU() { return u_.data(); }
    const oflow_tvl1_stats &stats() const { return st_; }

  private:
    void solve(const oflow_image &a, const oflow_image &b) {
        const oflow_flow f{u_.data(), u_.data() + (size_t)w_ * h_, 0, OFLOW_HOST};
        oflow::compat_check(oflow_tvl1(ctx_, &a, &b, &p_, &f, &st_), ctx_);
    }
    int w_, h_;
    oflow_tvl1_params p_{};
    oflow_ctx *ctx_ = nullptr;
    oflow_stream *stream_ = nullptr;
    std::vector<float> u_;
    oflow_tvl1_stats st_{};
};

// ------------------------------------------------------------------ Horn-Schunck
inline void initFlow(int nLevels, int stride, int width, int height) {
    if (nLevels < 1 || stride < width || height < 1)
        throw oflow::compat_error(OFLOW_ERR_BAD_ARG, "initFlow: bad arguments");
    oflow_ctx *&ctx = oflow::compat_global_ctx();
    if (!ctx) oflow::compat_check(oflow_ctx_create(0, &ctx), nullptr);
}

// Frames and flows are `height` rows of `stride` floats (flow.cuh:21-31).
inline void ComputeFlow(const float *I0, const float *I1, int width, int height, int stride,
                        float alpha, int nLevels, int nWarpIters, int nSolverIters, float *u,
                        float *v) {
    oflow_ctx *&ctx = oflow::compat_global_ctx();
    if (!ctx) oflow::compat_check(oflow_ctx_create(0, &ctx), nullptr);
    const oflow_image a{I0, width, height, stride, OFLOW_F32, OFLOW_HOST};
    const oflow_image b{I1, width, height, stride, OFLOW_F32, OFLOW_HOST};
    const oflow_hs_params p{alpha, nLevels, nWarpIters, nSolverIters};
    const oflow_flow f{u, v, stride, OFLOW_HOST};
    oflow::compat_check(oflow_hs(ctx, &a, &b, &p, &f), ctx);
}

inline void deleteFlow_mem(int /*nLevels*/) {
    oflow_ctx *&ctx = oflow::compat_global_ctx();
    if (ctx) oflow_ctx_destroy(ctx);
    ctx = nullptr;
}

// ------------------------------------------------------------------ Lucas-Kanade
class LucasKanade {
  public:
    LucasKanade(int spac_filt_size_, int temp_filt_size_, int window_size_, int nx_, int ny_,
                int device = 0)
        : nx(nx_), ny(ny_), ring((size_t)temp_filt_size_ * nx_ * ny_, 0) {
        p_.spac = spac_filt_size_;
        p_.temp = temp_filt_size_;
        p_.window = window_size_;
        p_.levels = 1;
        p_.iters = 1;
        oflow::compat_check(oflow_ctx_create(device, &ctx_), nullptr);
    }
    ~LucasKanade() { oflow_ctx_destroy(ctx_); }
    LucasKanade(const LucasKanade &) = delete;
    LucasKanade &operator=(const LucasKanade &) = delete;

    // Newest frame into ring slot fr % temp_size (kernels.cu:6-10).
    void copy_frames_circularbuffer_GPU_wrapper(unsigned char *frame, int temp_size, int fr,
                                                int frame_size) {
        if (temp_size != p_.temp || frame_size != nx * ny)
            throw oflow::compat_error(OFLOW_ERR_BAD_ARG, "ring or frame size mismatch");
        std::memcpy(ring.data() + (size_t)(fr % temp_size) * frame_size, frame, frame_size);
    }
    // Flow with the newest frame in slot iframe % temp (lucaskanade.cu:54-71).
    void lucas_kanade(float *Vx, float *Vy, int iframe) {
        std::vector<oflow_image> fr(p_.temp);
        for (int k = 0; k < p_.temp; k++)
            fr[k] = oflow_image{ring.data() + (size_t)k * nx * ny, nx, ny, 0, OFLOW_U8, OFLOW_HOST};
        const oflow_flow f{Vx, Vy, 0, OFLOW_HOST};
        oflow::compat_check(oflow_lk(ctx_, fr.data(), iframe, &p_, &f), ctx_);
    }

  private:
    int nx, ny;
    std::vector<unsigned char> ring;
    oflow_lk_params p_{};
    oflow_ctx *ctx_ = nullptr;
};

// ------------------------------------------------------------------ visualisation
// App::flowToColor (src/tvl1/sequential/main.cpp:93) with the cv::Mat output
// replaced by a caller buffer of width * height * 3 bytes (B, G, R).  flowData
// is the planar [u | v] layout of TV_L1::getU().
inline void flowToColor(int width, int height, const float *flowData, unsigned char *outBGR) {
    oflow_ctx *&ctx = oflow::compat_global_ctx();
    if (!ctx) oflow::compat_check(oflow_ctx_create(0, &ctx), nullptr);
    const oflow_flow f{const_cast<float *>(flowData), const_cast<float *>(flowData) + (size_t)width * height,
                       0, OFLOW_HOST};
    const oflow_bgr_image o{outBGR, 0, OFLOW_HOST};
    oflow::compat_check(oflow_flow_to_color(ctx, 1, width, height, &f, &o), ctx);
}

#endif  // OFLOW_COMPAT_HPP
