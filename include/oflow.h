/*
 * oflow -- dense optical flow (TV-L1, Horn-Schunck, Lucas-Kanade) on NVIDIA
 * B200 (sm_100a).  Thin C ABI: plain pointers, sizes and status codes; no
 * exceptions cross it and nothing in it exits the process.
 *
 * Each solver entry point takes two grayscale frames and the solver
 * parameters and returns a dense flow field (u = horizontal, v = vertical
 * displacement of a frame-0 pixel into frame 1).  It replaces these
 * reference interfaces (paths relative to the reference project root):
 *
 *   oflow_tvl1      TV_L1::TV_L1 + TV_L1::runDualTVL1Multiscale + TV_L1::getU
 *                   src/tvl1/sequential/tvl1.hpp:12-17 (uint8 frames) and
 *                   src/tvl1/cuda/tvl1.cuh:12-20 (float frames, streaming)
 *   oflow_hs        initFlow / ComputeFlow / deleteFlow_mem
 *                   src/hs/cuda/flow.cuh:19-33
 *   oflow_lk        LucasKanade::LucasKanade / copy_frames_circularbuffer_GPU_wrapper
 *                   / lucas_kanade, src/lk/cuda/lucaskanade.cuh:6-12
 *   oflow_pyrlk     pyramidal, iterated LK (no reference entry point; built from
 *                   the steps of src/lk/cuda/kernels/kernels.cu)
 *
 * Threading: a context is used by one host thread at a time; contexts are
 * independent.  Calls are synchronous (they return when the flow is in the
 * caller's buffers) unless a stream was set with oflow_ctx_set_stream and the
 * outputs are device buffers, in which case the call returns once the work is
 * enqueued on that stream.
 */
#ifndef OFLOW_H
#define OFLOW_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OFLOW_ABI_VERSION 1
#define OFLOW_MAX_SCALES 16
#define OFLOW_MAX_WARPS 32

typedef enum {
    OFLOW_OK = 0,
    OFLOW_ERR_BAD_ARG = 1,     /* invalid sizes, pointers or parameters */
    OFLOW_ERR_CUDA = 2,        /* CUDA runtime error (message via oflow_ctx_last_error) */
    OFLOW_ERR_TIMEOUT = 3,     /* a bounded device-side wait gave up */
    OFLOW_ERR_NO_DEVICE = 4,   /* no usable CUDA device */
    OFLOW_ERR_OOM = 5,         /* device allocation failed */
    OFLOW_ERR_UNSUPPORTED = 6  /* valid request outside what this build supports */
} oflow_status;

typedef enum { OFLOW_U8 = 0, OFLOW_F32 = 1 } oflow_dtype;
typedef enum { OFLOW_HOST = 0, OFLOW_DEVICE = 1 } oflow_location;

typedef struct oflow_ctx oflow_ctx;

/* A grayscale frame.  pitch is in elements (0 means width). */
typedef struct {
    const void *data;
    int width, height, pitch;
    int dtype;    /* oflow_dtype */
    int location; /* oflow_location */
} oflow_image;

/* Output flow planes, caller-owned.  pitch in elements (0 means width). */
typedef struct {
    float *u;
    float *v;
    int pitch;
    int location; /* oflow_location */
} oflow_flow;

/* ------------------------------------------------------------------ context */
oflow_status oflow_ctx_create(int device, oflow_ctx **out);
/* Waits for the context's work and frees it.  Nets and streams created on it
 * become inert: they can still be destroyed (and nothing else). */
oflow_status oflow_ctx_destroy(oflow_ctx *ctx);
/* Run subsequent work on a caller-owned cudaStream_t (NULL: the context's own
 * stream). */
oflow_status oflow_ctx_set_stream(oflow_ctx *ctx, void *cuda_stream);
/* Drop cached plans (device buffers and captured graphs). */
oflow_status oflow_ctx_trim(oflow_ctx *ctx);
const char *oflow_ctx_last_error(const oflow_ctx *ctx);
const char *oflow_status_string(int status);
int oflow_abi_version(void);

/* ------------------------------------------------------------------- TV-L1 */
/* Parameters of src/tvl1/sequential/tvl1.hpp:12-14 plus the inner-iteration
 * cap (tvl1.hpp:6).  Defaults: tau 0.25, lambda 0.15, theta 0.3, nscales 100
 * (then limited by the image size, tvl1.cpp:42-43), zfactor 0.5, warps 5,
 * epsilon 0.01, max_iterations 300. */
typedef struct {
    float tau, lambda, theta;
    int nscales;
    float zfactor;
    int warps;
    float epsilon;
    int max_iterations;
} oflow_tvl1_params;

/* Per-pair records of one solve.  iterations[s * warps + w] is the number of
 * inner iterations run at scale s (0 = finest), warp w. */
typedef struct {
    int nscales;
    int warps;
    int iterations[OFLOW_MAX_SCALES * OFLOW_MAX_WARPS];
    double energy; /* TV-L1 energy of the result (finest scale, last warp) */
} oflow_tvl1_stats;

void oflow_tvl1_default_params(oflow_tvl1_params *p);

/* Number of pyramid scales the solver will use for a w x h frame. */
int oflow_tvl1_nscales(int width, int height, const oflow_tvl1_params *p);

/* One frame pair.  stats may be NULL. */
oflow_status oflow_tvl1(oflow_ctx *ctx, const oflow_image *I0, const oflow_image *I1,
                        const oflow_tvl1_params *p, const oflow_flow *out,
                        oflow_tvl1_stats *stats);

/* n independent pairs in one schedule (sizes may differ).  Arrays of n.
 * stats may be NULL. */
oflow_status oflow_tvl1_batch(oflow_ctx *ctx, int n, const oflow_image *I0,
                              const oflow_image *I1, const oflow_tvl1_params *p,
                              const oflow_flow *out, oflow_tvl1_stats *stats);

/* Diagnostic form of oflow_tvl1: also records the TV-L1 energy (sum of |grad u|
 * over both components plus lambda * sum |rho(u)|, rho linearised at the
 * current warp) after the u update of every inner iteration, at
 * energy[(s * warps + w) * max_iterations + n]; entries past a stage's early
 * stop are left untouched.  energy holds nscales*warps*max_iterations doubles.
 * Slow (one extra reduction per iteration, no graph); for validation. */
oflow_status oflow_tvl1_energy_trace(oflow_ctx *ctx, const oflow_image *I0,
                                     const oflow_image *I1, const oflow_tvl1_params *p,
                                     const oflow_flow *out, oflow_tvl1_stats *stats,
                                     double *energy);

/* Timing of one solve, measured with CUDA events on the launching stream
 * around every warp and inner-iteration kernel (eager launches, no graph). */
typedef struct {
    double total_ms;       /* whole solve */
    double iter_ms;        /* sum over inner-iteration launches */
    double warp_ms;        /* sum over warp (bicubic resampling) launches */
    int iter_launches;
    int warp_launches;
    int launches;          /* all kernel launches of the schedule */
    double iter_ms_scale[OFLOW_MAX_SCALES]; /* inner-iteration time per scale */
} oflow_tvl1_profile;

/* Like oflow_tvl1_batch (outputs and stats included) with the timings above. */
oflow_status oflow_tvl1_batch_profile(oflow_ctx *ctx, int n, const oflow_image *I0,
                                      const oflow_image *I1, const oflow_tvl1_params *p,
                                      const oflow_flow *out, oflow_tvl1_stats *stats,
                                      oflow_tvl1_profile *prof);

/* Autotuner: solves the n given pairs (one size) once, then times every
 * inner-iteration configuration at every scale on the device and keeps the
 * fastest for plans of this size and batch: 0 = 64x32 tiles, 1 = 64x16,
 * 2 = 32x16, 3 = 16x8 (up to 4 iterations per launch), 4 = the whole level of
 * a pair in one block, 5 = the whole level in row bands over a cluster of 8
 * blocks (4 and 5 where the level fits shared memory).
 * cfg_per_scale (OFLOW_MAX_SCALES ints, may be NULL) receives the choice per
 * scale, -1 past the last scale.  The table lives in the context; it can be
 * saved to / loaded from a text file (lines: solver width height batch config)
 * keyed by the level size, so plans built later pick it up. */
oflow_status oflow_tvl1_autotune(oflow_ctx *ctx, int n, const oflow_image *I0,
                                 const oflow_image *I1, const oflow_tvl1_params *p,
                                 int *cfg_per_scale);
oflow_status oflow_ctx_save_tuning(oflow_ctx *ctx, const char *path);
/* Kernel launches the last oflow_tvl1 / oflow_tvl1_batch call of this context
 * executed on the device (the captured schedule: per warp ceil(max/4)+1
 * inner-iteration launches, those after every pair stopped returning at
 * once). */
oflow_status oflow_ctx_last_launches(oflow_ctx *ctx, long long *launches);
oflow_status oflow_ctx_load_tuning(oflow_ctx *ctx, const char *path);

/* Device check of the arithmetic behind the exact fast forms (no counterpart
 * in the reference; a diagnostic for tests and for new GPUs).  The TV-L1
 * kernels round exactly as IEEE single precision by refining the hardware's
 * reciprocal estimate; this runs that refinement on the device and counts
 * operands that break its contract:
 *   which 1: the refined reciprocal equal to __frcp_rn, bit patterns [lo, hi)
 *   which 3: Markstein's quotient from the refined reciprocal equal to IEEE
 *            division, seeded pseudo-random operands, indices [lo, hi)
 * (other values of which: OFLOW_ERR_BAD_ARG)
 * Synchronous on the default stream of the current device; *mismatches
 * receives the count (0 means the contract held on every operand). */
oflow_status oflow_selftest_math(int which, uint32_t lo, uint32_t hi, unsigned long long seed,
                                 unsigned long long *mismatches);

/* ------------------------------------------------------------ Horn-Schunck */
/* Parameters of ComputeFlow (src/hs/cuda/flow.cuh:21-31).  nlevels pyramid
 * levels (2x2 box downscale), nwarp warps per level, nsolver Jacobi sweeps. */
typedef struct {
    float alpha;
    int nlevels;
    int nwarp;
    int nsolver;
} oflow_hs_params;

void oflow_hs_default_params(oflow_hs_params *p);
oflow_status oflow_hs(oflow_ctx *ctx, const oflow_image *I0, const oflow_image *I1,
                      const oflow_hs_params *p, const oflow_flow *out);
oflow_status oflow_hs_batch(oflow_ctx *ctx, int n, const oflow_image *I0,
                            const oflow_image *I1, const oflow_hs_params *p,
                            const oflow_flow *out);
/* Autotuner for Horn-Schunck: solves the n given pairs (one size) once, then
 * times every Jacobi configuration (tile shape and sweeps per launch: 0 =
 * 32x16 tiles with 4 sweeps, 1 = 32x16 with 8, 2 = 64x32 with 8, 3 = 64x16
 * with 4, 4 = 32x32 with 16, 5 = 64x32 with 4) at every pyramid level and
 * keeps the fastest for
 * plans of this level size and batch (table entries with solver "hs", saved and
 * loaded with the TV-L1 ones).  cfg_per_level (OFLOW_MAX_SCALES ints, may be
 * NULL) receives the choice per level (coarsest first), -1 past the last.
 * Every configuration gives the same bits.  The reference has one fixed
 * configuration and no tuner. */
oflow_status oflow_hs_autotune(oflow_ctx *ctx, int n, const oflow_image *I0,
                               const oflow_image *I1, const oflow_hs_params *p,
                               int *cfg_per_level);

/* Horn-Schunck for callers that cannot allocate device memory: real-time
 * frame loops that cannot afford the device-wide synchronisation that
 * cudaMalloc/cudaFree may imply, and hosts that hand the library a fixed
 * memory budget up front.  This entry point has no counterpart in the
 * reference.
 *
 * It allocates nothing and needs no context.  Its scratch is one static
 * device array of 8 MiB, held by every GPU that loads the library until the
 * process exits.  With nlevels = 1 a frame needs 64 B per pixel (320x240:
 * 4.9 MB), so frames up to about 131,000 pixels fit; more levels add up to
 * 8/3 B per pixel for the pyramid.  Larger requests return OFLOW_ERR_BAD_ARG.
 * I0, I1 are device float frames, u and v device float planes; pitches are in
 * elements (0 means width).  The work is enqueued on `stream` (a
 * cudaStream_t; NULL is the default stream) and the call returns without
 * waiting.  The result equals oflow_hs with the same parameters.
 *
 * The first call on a device looks up the array's device address (with that
 * device current) and caches it for the process; make that first call before
 * any stream capture.  The cached address does not survive a device reset
 * (cudaDeviceReset, or the primary context being destroyed and recreated):
 * do not call this entry point on a device after such a reset.  All calls
 * share the one array, which keeps the last call's contents: calls that
 * overlap on the GPU (on different streams, or from several threads without
 * ordering) race and give wrong results.  Order them on one stream. */
oflow_status oflow_hs_noalloc(const float *I0, const float *I1, int width, int height,
                              int pitch, const oflow_hs_params *p, float *u, float *v,
                              int out_pitch, void *stream);

/* ------------------------------------------------------------ mixed batches */
typedef enum { OFLOW_SOLVER_TVL1 = 0, OFLOW_SOLVER_HS = 1 } oflow_solver;

/* One frame pair of a mixed batch. */
typedef struct {
    int solver;                     /* oflow_solver */
    oflow_image I0, I1;
    const oflow_tvl1_params *tvl1;  /* used when solver == OFLOW_SOLVER_TVL1 */
    const oflow_hs_params *hs;      /* used when solver == OFLOW_SOLVER_HS */
    oflow_flow out;
} oflow_job;

/* Solves n pairs of mixed solvers and sizes as one schedule: the pairs are
 * grouped by (solver, size, dtype, parameters), each group is a batched plan,
 * and all groups' launch sequences are captured into one CUDA graph as
 * parallel branches, so groups run concurrently on the device.  The graph is
 * kept for the batch composition and replayed when the same composition
 * comes again. */
oflow_status oflow_batch(oflow_ctx *ctx, int n, const oflow_job *jobs);

/* --------------------------------------------------- learned warm start (TV-L1) */
/* A small encoder-decoder network (4 stages, 32/64/96/128 channels, 3x3
 * convolutions, BF16 weights and activations, FP32 accumulation on tensor
 * cores) that predicts flow at 1/8 resolution -- the size of TV-L1 scale 3 --
 * from a frame pair.  No counterpart in the reference.  One network object
 * serves `batch` pairs of width x height per call. */
typedef struct oflow_net oflow_net;
int oflow_net_num_params(void);
oflow_status oflow_net_create(oflow_ctx *ctx, int width, int height, int batch, oflow_net **out);
oflow_status oflow_net_destroy(oflow_net *net);
oflow_status oflow_net_out_size(const oflow_net *net, int *width, int *height);
/* fp32 parameters (per layer: weights [K][3][3][C], then bias), host memory */
oflow_status oflow_net_set_params(oflow_net *net, const float *params);
oflow_status oflow_net_get_params(oflow_net *net, float *params);
/* frames: device buffer [batch][2][height][width] (dtype OFLOW_U8 / OFLOW_F32);
 * target: device f32 [batch][out_h][out_w][2].  One Adam step on the
 * Charbonnier loss; *loss receives the mean loss before the step. */
oflow_status oflow_net_train_step(oflow_net *net, const void *frames, int dtype,
                                  const float *target, float lr, double *loss);
/* flow: device f32 [batch][out_h][out_w][2] */
oflow_status oflow_net_predict(oflow_net *net, const void *frames, int dtype, float *flow);

/* TV-L1 warm-started by the network: the network's flow initialises scale 3
 * and the solve runs scales 3..0 with `warm` (e.g. 2 warps x 20 iterations),
 * or per scale with warps_per_scale[s] (in [1, warm->warps]) and
 * iters_per_scale[s] for s = 0 (finest) .. 3; either array may be NULL for
 * the uniform value of `warm`, and entries beyond scale 3 are ignored.
 * With `plain` non-NULL the plain solve also runs and is the judge: a pair's
 * warm result is kept only if (a) its TV-L1 energy (non-linearised: sum
 * |grad u| + lambda * sum |I1(x+u) - I0(x)|, bicubic warp with border zeroing)
 * is at most 1.01 times the plain solve's, and (b) its end-point difference
 * from the plain flow, summed over the pixels, is at most 1 % of the plain
 * flow's summed magnitude; otherwise the plain result is returned.
 * n must equal the network's batch and all frames its size.  energy_warm,
 * energy_plain, epe_vs_plain (the ratio of (b)), accepted and stats (arrays
 * of n; stats = the warm solve's iterations per (scale, warp), 0 for the
 * scales above 3) may be NULL. */
oflow_status oflow_tvl1_warm(oflow_ctx *ctx, oflow_net *net, int n, const oflow_image *I0,
                             const oflow_image *I1, const oflow_tvl1_params *warm,
                             const int *warps_per_scale, const int *iters_per_scale,
                             const oflow_tvl1_params *plain, const oflow_flow *out,
                             double *energy_warm, double *energy_plain, double *epe_vs_plain,
                             int *accepted, oflow_tvl1_stats *stats);

/* ---------------------------------------------------------------- streaming */
/* Frame streams: the streaming form of the reference's CUDA TV-L1
 * (runDualTVL1Multiscale(const float *I), src/tvl1/cuda/tvl1.cu:122-130) --
 * each new frame is paired with the previous one, which stays in device
 * memory, so a frame crosses the bus once.  A stream carries `lanes`
 * independent videos of one size and solver; one push takes one new frame per
 * lane and solves all lanes' pairs (previous, new) as one batch.  Before a
 * lane's first frame its previous frame is all zeros (the reference's
 * buffer before its first call).  Uploads run on the stream's own copy
 * stream: once a push's solve has taken its frames, the next push's upload
 * overlaps the rest of that solve (pinned host frames, or device frames, and
 * a stream set with oflow_ctx_set_stream with device outputs, make pushes
 * asynchronous; otherwise a push returns with the flow in place). */
typedef struct oflow_stream oflow_stream;
typedef struct {
    int solver; /* OFLOW_SOLVER_TVL1 or OFLOW_SOLVER_HS */
    int width, height;
    int dtype;  /* of the frames pushed: OFLOW_U8 or OFLOW_F32 */
    int lanes;  /* videos per stream, >= 1 */
    oflow_tvl1_params tvl1;
    oflow_hs_params hs;
} oflow_stream_desc;
oflow_status oflow_stream_create(oflow_ctx *ctx, const oflow_stream_desc *desc, oflow_stream **out);
oflow_status oflow_stream_destroy(oflow_stream *s);
/* frames, out: arrays of `lanes`; stats (TV-L1, array of lanes) may be NULL */
oflow_status oflow_stream_push(oflow_stream *s, const oflow_image *frames, const oflow_flow *out,
                               oflow_tvl1_stats *stats);
/* frames pushed so far */
long long oflow_stream_frames(const oflow_stream *s);

/* ------------------------------------------------------------ visualisation */
/* An 8-bit, 3-channel image (bytes B, G, R per pixel), caller-owned.  pitch in
 * bytes (0 means 3 * width). */
typedef struct {
    uint8_t *data;
    int pitch;
    int location; /* oflow_location */
} oflow_bgr_image;

/* The demos' flowToColor (App::flowToColor, src/tvl1/sequential/main.cpp:
 * 93-126) for n flows of width x height: V = 8-bit min(10 |(u,v)|, 255),
 * H = 8-bit atan2(v, u) in degrees / 2 (negative angles saturate to 0),
 * S = 255, converted HSV -> B, G, R (hexcone, H in 0..180) into out[i] instead
 * of an OpenCV window.  Flows and images may each be host or device buffers;
 * the call is synchronous unless a stream was set and everything is on the
 * device. */
oflow_status oflow_flow_to_color(oflow_ctx *ctx, int n, int width, int height,
                                 const oflow_flow *flows, const oflow_bgr_image *out);

/* One product of a 3x3 convolution (pad 1, stride 1 or 2) on device buffers,
 * for validating the network's kernels.  mode 0: y = conv(x, w) + bias (ReLU if
 * relu; y f32 if out_f32 else bf16) on the tcgen05 tensor-core kernel the
 * network's forward pass uses (C % 16 == 0, K <= 128; OFLOW_ERR_TIMEOUT if one
 * of its bounded waits gave up); mode 3: the same product on the mma.sync
 * kernel; mode 1: gin = conv^T(g) (f32; g masked by y_act > 0 when y_act is
 * non-NULL) on the tcgen05 kernel, as a forward convolution of the masked
 * gradient with rotated weights (C % 16 == 0, K % 8 == 0; K is padded to a
 * multiple of 16 with zero channels); mode 4: the same product on the mma.sync
 * kernel; mode 2: gw = dL/dw, gbias = dL/db (f32) on the tcgen05 kernel
 * (C % 16 == 0, K % 8 == 0, K <= 128); mode 5: the same on the
 * mma.sync kernel.  x, w, y_act: bf16; g: f32.  Shapes: x [N,H,W,C],
 * w [K,3,3,C], y [N,P,Q,K]. */
oflow_status oflow_conv3x3(int mode, int N, int H, int W, int C, int K, int stride, int relu,
                           int out_f32, const void *x_or_g, const void *y_act, const void *w_or_x,
                           void *out, const float *bias, float *gbias, void *stream);

/* ------------------------------------------------------------ Lucas-Kanade */
/* spac: spatial derivative taps (1,3,5,7,9); temp: temporal taps
 * (1,2,3,5,7,9); window: odd window side (src/lk/cuda/lucaskanade.cuh:8).
 * levels/iters are used by oflow_pyrlk only. */
typedef struct {
    int spac;
    int temp;
    int window;
    int levels;
    int iters;
} oflow_lk_params;

void oflow_lk_default_params(oflow_lk_params *p);

/* Single-step LK over a ring of `temp` uint8 frames: frames[k] is ring slot k,
 * and the newest frame sits in slot iframe % temp (the reference keeps the
 * ring on the device and fills slot fr % temp, kernels.cu:6-10).  The spatial
 * derivatives are taken on the oldest frame of the ring. */
oflow_status oflow_lk(oflow_ctx *ctx, const oflow_image *frames, int iframe,
                      const oflow_lk_params *p, const oflow_flow *out);

/* Pyramidal, iterated LK on two frames (levels at scale 0.5, `iters`
 * warp-and-solve refinements per level, temporal taps (-1, 1)). */
oflow_status oflow_pyrlk(oflow_ctx *ctx, const oflow_image *I0, const oflow_image *I1,
                         const oflow_lk_params *p, const oflow_flow *out);

/* n pairs in one call (no reference entry point; the batched form of
 * oflow_pyrlk for many small frames, which one pair cannot spread over the
 * GPU).  Pairs of one size and dtype share one plan and one CUDA graph; each
 * flow equals oflow_pyrlk's on the same pair. */
oflow_status oflow_pyrlk_batch(oflow_ctx *ctx, int n, const oflow_image *I0,
                               const oflow_image *I1, const oflow_lk_params *p,
                               const oflow_flow *out);

#ifdef __cplusplus
}
#endif

#endif /* OFLOW_H */
