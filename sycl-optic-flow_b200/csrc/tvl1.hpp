// Batched TV-L1 plan: device buffers for B equal-size pairs and the captured
// schedule (ingest, normalisation, pyramid, coarse-to-fine warps and inner
// iterations, output split).
#pragma once

#include <cuda.h>

#include <map>
#include <tuple>

#include "internal.hpp"

#include <vector>

namespace oflow {

// Normalised Gaussian half-kernel (centre + radius taps), double precision.
struct GaussTaps {
    double B[16];
    int size;  // taps including the centre; radius = size - 1
};

int tvl1_nscales(int w, int h, int nscales, float zfactor);

// Tuned kernel configurations: key (solver, level w, level h, batch) -> config index.
using TuneKey = std::tuple<int, int, int, int>;
using TuneTable = std::map<TuneKey, int>;
enum { kTuneTvl1 = 1, kTuneHs = 2 };
inline TuneKey tune_key(int w, int h, int B, int solver = kTuneTvl1) {
    return TuneKey(solver, w, h, B);
}
void tvl1_zoom_size(int nx, int ny, int *nxx, int *nyy, float f);
// Taps of the pre-decimation blur, sigma = 0.6*sqrt(1/f^2 - 1) (zoom.cpp:39).
GaussTaps make_zoom_taps(float zfactor);
// Separable Gaussian of `planes` dense nx*ny planes (stride apart), src -> dst.
void launch_gauss(const float *src, float *dst, int nx, int ny, size_t stride,
                  const GaussTaps &t, int planes, cudaStream_t st);
// Bicubic resample (no border zeroing) at ((float)j/dx, (float)i/dy).
void launch_resample(const float *src, size_t sstride, int nx, int ny, float *dst,
                     size_t dstride, int nxx, int nyy, float dx, float dy, int planes,
                     cudaStream_t st);
// zoom_out of `planes` planes (zoom.cpp:20-53): blur with `t` then resample by
// zfactor.  At zfactor 1/2 one fused pass (T unused), otherwise blur into the
// scratch planes T (stride sstride) and resample.  Returns the launch count.
int launch_zoom_out(const float *src, size_t sstride, int nx, int ny, float *T, float *dst,
                    size_t dstride, int nxx, int nyy, float zfactor, const GaussTaps &t,
                    int planes, cudaStream_t st);

// A tiled TMA map of 8-byte elements with zero fill outside (dims innermost
// first, byte strides of dims 1..rank-1, box per dim); false if the driver
// refuses it (the caller then loads with plain instructions).
bool encode_map8(CUtensorMap *m, void *base, int rank, const cuuint64_t *dims,
                 const cuuint64_t *strides, const cuuint32_t *box);

// Column coefficients of the warp's bicubic samples at one level, per texel
// of every pair: (c3, c2) of I1, I1x and I1y in double, and (v2 - v0, v1) of
// each in single precision (I1 and I1x in dv01, I1y in dv2).
struct WarpCoef {
    double2 *cc0, *cc1, *cc2;
    float4 *dv01;
    float2 *dv2;
};

// Where a plan reads one input frame: a device pointer of the plan's dtype and
// its row pitch in elements.
struct FrameRef {
    const void *p;
    long long pitch;
};

// Where a plan writes one pair's flow: u and v planes, row pitch in elements.
struct OutRef {
    float *u;
    float *v;
    long long pitch;
};

class TvPlan {
  public:
    // start_scale >= 0: warm start -- the solve begins at that scale from the
    // flow written into uz() (in that scale's pixel units) instead of zero at
    // the coarsest scale.
    TvPlan(int w, int h, int B, int dtype, const oflow_tvl1_params &prm, bool trace = false,
           const TuneTable *tuned = nullptr, int start_scale = -1);
    float2 *uz() const;
    size_t plane_stride() const { return N0_; }
    int start_scale() const { return s0_; }
    // Non-linearised TV-L1 energy of the last result, per pair (see
    // k_energy_true): sum |grad u1| + |grad u2| + lambda * sum |I1(x+u) - I0(x)|.
    void true_energy(double *host_out, cudaStream_t st);
    // Per pair: sum of end-point differences of this plan's last flows against
    // `other`'s (same shape), over the sum of `other`'s flow magnitudes.
    // Synchronises.
    void rel_epe_against(const TvPlan &other, double *host_out, cudaStream_t st);
    // Times each blocked-iteration configuration per scale on the current
    // buffers, keeps the fastest and records it in `table`.
    void autotune(cudaStream_t st, TuneTable *table, int reps = 3);
    int tb_config(int s) const { return tb_cfg_[s]; }
    // Per-scale schedule (index 0 = finest) of the scales the plan solves (0
    // to its start scale; entries above are ignored): warps in [1,
    // params.warps] and iteration caps; nullptr keeps the parameters' uniform
    // value.  Rebuilds the graph on change.  Not for traced plans.
    void set_schedule(const int *warps, const int *iters);
    bool same_schedule(const int *warps, const int *iters) const;
    // Tiled warp stages as one persistent work-queue launch each (default) or
    // as one launch per block of K iterations (for plans that share the GPU
    // with concurrent kernels).  Same results either way.
    void use_queue(bool on) {
        if (on != queue_) graph_.reset();
        queue_ = on && !queue_off_env_;
    }
    // The plan runs beside parts - 1 others of its kind on the GPU (the
    // chunks of a host batch): its persistent launches take that fraction of
    // the resident slots.
    void set_share(int parts) {
        if (parts != share_) graph_.reset();
        share_ = parts < 1 ? 1 : parts;
    }
    // Device destination of input frame k (0: I0, 1: I1) of pair b: a dense
    // w*h plane of the plan's dtype.
    void *raw_input(int b, int k) const;
    // The next run reads frame k of pair b straight from `p` (device, the
    // plan's dtype, `pitch` elements per row) instead of raw_input(b, k);
    // bind_raw restores the staging buffer.  The table is uploaded by run(),
    // run_eager() and profile().
    void bind_frame(int b, int k, const void *p, int pitch);
    void bind_raw(int b, int k);
    // Flow of pair b: the caller's device planes (written in place by the
    // schedule's last kernel; pitch in elements, 0 = width) or this plan's
    // output buffer (out_u / out_v).  Plans start with their own buffers.
    void bind_out(int b, float *u, float *v, int pitch);
    void bind_own_out(int b);
    const float *out_u(int b) const;
    const float *out_v(int b) const;
    const int *iters_dev() const;
    // Enqueue the whole solve (captured into a graph on first use).
    void run(cudaStream_t st);
    // Enqueue the launches directly on `st` (also what the graph captures);
    // reads the frame table as last uploaded.
    void record(cudaStream_t st);
    // upload the frame table, then record(): an eager run
    void run_eager(cudaStream_t st);
    // The final energy (k_energy) of the last run's result, per pair, for
    // read_stats; enqueue once after run() when statistics are wanted (traced
    // plans compute it in their schedule).
    void compute_energy(cudaStream_t st);
    void read_stats(int b, oflow_tvl1_stats *out, cudaStream_t st) const;
    // Eager run with events around each warp / inner-iteration launch.
    void profile(cudaStream_t st, oflow_tvl1_profile *out);
    int launches() const { return launches_; }
    // kernel launches of one graph replay (run()): the fixed schedule, whose
    // launches after every pair of a warp stage stopped return at once
    long long device_launches(cudaStream_t) const { return graph_launches_; }
    void read_energy_trace(int b, double *dst, cudaStream_t st) const;

    int width() const { return w_; }
    int height() const { return h_; }
    int batch() const { return B_; }
    int dtype() const { return dtype_; }
    int nscales() const { return ns_; }
    int level_w(int s) const { return nx_[s]; }
    int level_h(int s) const { return ny_[s]; }
    int energy_slots() const { return energy_slots_; }
    bool traced() const { return trace_; }
    const oflow_tvl1_params &params() const { return prm_; }
    size_t device_bytes() const { return ar_.size(); }
    // Throws OFLOW_ERR_TIMEOUT if a kernel of this plan gave up a bounded wait
    // (a tile's TMA load) since the last check; reads host memory only.
    void check_device_error();

  private:
    int w_, h_, B_, dtype_;
    oflow_tvl1_params prm_;
    bool trace_;
    int ns_ = 0;
    int nx_[OFLOW_MAX_SCALES] = {}, ny_[OFLOW_MAX_SCALES] = {};
    size_t pyr_off_[OFLOW_MAX_SCALES] = {};
    size_t N0_ = 0;
    int iter_blocks_ = 0, ingest_blocks_ = 0, energy_blocks_ = 0, max_blocks_ = 0;
    int iter_stride_ = 0, energy_slots_ = 0;
    GaussTaps taps0_{}, tapsz_{};
    struct Prof {
        std::vector<cudaEvent_t> ev;  // begin/end pairs
        std::vector<int> tag;         // per pair: -1 warp launch, else the scale
        int n_ev = 0;
    };
    Prof *prof_ = nullptr;
    int launches_ = 0;
    Arena ar_;
    int tb_cfg_[OFLOW_MAX_SCALES] = {};
    int s0_ = 0;
    bool warm_ = false;
    size_t o_tarr_ = 0, o_tout_ = 0;
    int sw_[OFLOW_MAX_SCALES] = {}, si_[OFLOW_MAX_SCALES] = {};  // warps, iterations per scale
    size_t o_WR_ = 0;
    size_t o_raw_ = 0, o_T_ = 0, o_pyr_ = 0, o_cc_ = 0, o_U0_ = 0, o_Uz_ = 0, o_P0_ = 0,
           o_out_ = 0, o_ctrl_ = 0, o_part_ = 0, o_recs_ = 0, o_iters_ = 0, o_energy_ = 0;
    float2 *ubuf(int k) const;  // state buffer k of u (all pairs)
    float4 *pbuf(int k) const;  // state buffer k of p
    Graph graph_;
    int graph_launches_ = 0;
    std::vector<FrameRef> frames_;  // [B][2], host copy of the device table
    HostFlag err_;
    size_t o_frames_ = 0;
    size_t o_queue_ = 0, o_left_ = 0, o_otab_ = 0;
    std::vector<OutRef> outs_;  // [B], host copy of the device output table
    bool queue_ = true;  // tiled stages as one persistent launch each
    bool queue_off_env_ = false;
    int predict_ = 2;  // queue form: blocks of iterations end at the predicted stop
    int share_ = 1;    // fraction (1/share_) of the resident slots a queue launch takes

  public:
    // the frame and output tables to the device (run() does it; a caller that
    // records the schedule into its own graph does it before each launch)
    void upload_frames(cudaStream_t st);
};

}  // namespace oflow
