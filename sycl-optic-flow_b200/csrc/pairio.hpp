// Where a batched plan reads its frames and writes its flows: two small
// tables in device memory that the captured schedule reads on every run.
// Each entry points either at the plan's own staging / output buffers (host
// frames and flows pass through those) or at the caller's device buffers,
// which the kernels then read and write in place, with no copy per pair.
#pragma once

#include <vector>

#include "internal.hpp"
#include "tvl1.hpp"

namespace oflow {

class PairIo {
  public:
    // dev_frames: 2*B entries (pair b, frame k at 2b+k); dev_outs: B entries
    void init(FrameRef *dev_frames, OutRef *dev_outs, int B) {
        df_ = dev_frames;
        do_ = dev_outs;
        frames_.assign(2 * (size_t)B, FrameRef{nullptr, 0});
        outs_.assign((size_t)B, OutRef{nullptr, nullptr, 0});
    }
    void set_frame(int b, int k, const void *p, long long pitch) { frames_[2 * (size_t)b + k] = FrameRef{p, pitch}; }
    void set_out(int b, float *u, float *v, long long pitch) { outs_[b] = OutRef{u, v, pitch}; }
    // both tables, on `st` (pageable sources: copied out before returning)
    void upload(cudaStream_t st) const {
        OF_CUDA(cudaMemcpyAsync(df_, frames_.data(), sizeof(FrameRef) * frames_.size(),
                                cudaMemcpyHostToDevice, st));
        OF_CUDA(cudaMemcpyAsync(do_, outs_.data(), sizeof(OutRef) * outs_.size(),
                                cudaMemcpyHostToDevice, st));
    }
    const FrameRef *frames() const { return df_; }
    const OutRef *outs() const { return do_; }

  private:
    FrameRef *df_ = nullptr;
    OutRef *do_ = nullptr;
    std::vector<FrameRef> frames_;
    std::vector<OutRef> outs_;
};

// Level-0 float planes from the frame table: plane z (= 2b+k) at dst + z*N,
// rows of w (u8 or f32 frames, any row pitch).
void launch_ingest_tab(const FrameRef *frames, int dtype, int w, int h, float *dst, size_t N,
                       int planes, cudaStream_t st);
// Flow (u, v) of pair b (U + b*stride, rows of w) into the output table.
void launch_split_tab(const float2 *U, size_t stride, int w, int h, const OutRef *outs, int B,
                      cudaStream_t st);

}  // namespace oflow
