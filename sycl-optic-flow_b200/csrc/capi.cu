// The C ABI (include/oflow.h): contexts, plan caches, staging of frames and
// flows, and the status-code boundary.  Nothing here throws across the ABI or
// exits the process; CUDA errors come back as OFLOW_ERR_CUDA with the message
// kept in the context.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "color.hpp"
#include "hs.hpp"
#include "internal.hpp"
#include "lk.hpp"
#include "tvl1.hpp"
#include "warmnet.hpp"

using namespace oflow;

namespace oflow {

size_t dtype_size(int dtype) { return dtype == OFLOW_U8 ? 1 : 4; }

void check_image(const oflow_image *img, const char *name) {
    OF_CHECK(img != nullptr, std::string(name) + ": null image");
    OF_CHECK(img->data != nullptr, std::string(name) + ": null data pointer");
    OF_CHECK(img->width > 0 && img->height > 0, std::string(name) + ": empty image");
    OF_CHECK(img->dtype == OFLOW_U8 || img->dtype == OFLOW_F32, std::string(name) + ": bad dtype");
    OF_CHECK(img->location == OFLOW_HOST || img->location == OFLOW_DEVICE,
             std::string(name) + ": bad location");
    OF_CHECK(img->pitch == 0 || img->pitch >= img->width, std::string(name) + ": pitch < width");
}

static void check_flow(const oflow_flow *f, int w) {
    OF_CHECK(f != nullptr && f->u != nullptr && f->v != nullptr, "output: null flow pointer");
    OF_CHECK(f->location == OFLOW_HOST || f->location == OFLOW_DEVICE, "output: bad location");
    OF_CHECK(f->pitch == 0 || f->pitch >= w, "output: pitch < width");
}

void stage_image(const oflow_image &img, void *dst, size_t elem, cudaStream_t s) {
    const size_t spitch = (size_t)(img.pitch ? img.pitch : img.width) * elem;
    const size_t row = (size_t)img.width * elem;
    OF_CUDA(cudaMemcpy2DAsync(dst, row, img.data, spitch, row, img.height,
                              img.location == OFLOW_HOST ? cudaMemcpyHostToDevice
                                                         : cudaMemcpyDeviceToDevice,
                              s));
}

void unstage_plane(const float *src, int w, int h, float *dst, int pitch, int loc,
                   cudaStream_t s) {
    const size_t row = (size_t)w * 4, dpitch = (size_t)(pitch ? pitch : w) * 4;
    OF_CUDA(cudaMemcpy2DAsync(dst, dpitch, src, row, row, h,
                              loc == OFLOW_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                              s));
}

// Stages a pair into the plan's own buffers and points its frame table there;
// its flow goes to the plan's own output buffer (the caller reads it there).
void stage_pair_raw(TvPlan &pl, int b, const oflow_image &I0, const oflow_image &I1, cudaStream_t s) {
    stage_image(I0, pl.raw_input(b, 0), dtype_size(I0.dtype), s);
    stage_image(I1, pl.raw_input(b, 1), dtype_size(I1.dtype), s);
    pl.bind_raw(b, 0);
    pl.bind_raw(b, 1);
    pl.bind_own_out(b);
}

}  // namespace oflow

namespace {
// A mixed batch: one plan per (solver, size, dtype, parameters) group and one
// graph with a parallel branch per group.
struct MixedBatch {
    std::vector<std::string> key;
    std::vector<std::vector<int>> members;  // job indices per group
    std::vector<std::unique_ptr<TvPlan>> tv;
    std::vector<std::unique_ptr<HsPlan>> hs;
    std::vector<int> kind, slot;            // per group: solver and index into tv/hs
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> events;
    Graph graph;
    ~MixedBatch() {
        for (auto s : streams) cudaStreamDestroy(s);
        for (auto e : events) cudaEventDestroy(e);
    }
};
}  // namespace

// A TV-L1 batch with frames or flows in host memory may be solved in up to
// this many chunks, each a plan of its own on a side stream, so that the
// copies of one chunk overlap the solves of the others (OFLOW_HOST_CHUNKS).
// By default it is one plan with its copies before and after: for 32 pairs of
// 1024x436 that measured 1,155 pairs/s end to end against 1,143 with four
// concurrent chunks (one launch per block of iterations) and 778-986 with the
// chunks' solves one after another, each with the work queue (a small plan
// pays the latency-bound coarse scales again).
constexpr int kHostChunks = 4;
constexpr int kChunkMinPairs = 4;

struct oflow_ctx {
    int device = 0;
    cudaStream_t own = nullptr;
    cudaStream_t user = nullptr;
    std::string err;
    std::vector<std::unique_ptr<TvPlan>> tv;
    std::vector<std::unique_ptr<HsPlan>> hs;
    std::vector<std::unique_ptr<PyrLkPlan>> pyrlk;
    std::vector<std::unique_ptr<LkPlan>> lk;
    TuneTable tune;  // autotuned kernel configurations, consulted by new plans
    std::vector<std::unique_ptr<TvPlan>> tv_warm;  // plans that start at scale 3
    std::vector<std::unique_ptr<MixedBatch>> mixed;
    DevBuf color_scratch;  // host-side flows / images of oflow_flow_to_color
    std::vector<TvPlan *> last_tv;  // plans run by the last oflow_tvl1(_batch) call
    // objects created on this context; destroying the context detaches them
    std::vector<oflow_net *> nets;
    std::vector<oflow_stream *> streams;
    // chunked host solves: one plan cache and one stream per chunk slot
    std::vector<std::unique_ptr<TvPlan>> tv_side[kHostChunks];
    cudaStream_t side[kHostChunks] = {};
    cudaEvent_t fork = nullptr, join[kHostChunks] = {};
    cudaStream_t stream() const { return user ? user : own; }
};

namespace {

constexpr size_t kMaxPlans = 8;

template <typename P> void keep_recent(std::vector<std::unique_ptr<P>> &v) {
    while (v.size() > kMaxPlans) v.erase(v.begin());
}

bool same(const oflow_tvl1_params &a, const oflow_tvl1_params &b) {
    return std::memcmp(&a, &b, sizeof(a)) == 0;
}
bool same(const oflow_hs_params &a, const oflow_hs_params &b) {
    return std::memcmp(&a, &b, sizeof(a)) == 0;
}
bool same(const oflow_lk_params &a, const oflow_lk_params &b) {
    return std::memcmp(&a, &b, sizeof(a)) == 0;
}

template <typename F> oflow_status guard(oflow_ctx *ctx, F &&f) {
    try {
        if (ctx) OF_CUDA(cudaSetDevice(ctx->device));
        f();
        if (ctx) ctx->err.clear();
        return OFLOW_OK;
    } catch (const Error &e) {
        if (ctx) ctx->err = e.what();
        return e.code;
    } catch (const std::bad_alloc &) {
        if (ctx) ctx->err = "host allocation failed";
        return OFLOW_ERR_OOM;
    } catch (const std::exception &e) {
        if (ctx) ctx->err = e.what();
        return OFLOW_ERR_CUDA;
    } catch (...) {
        if (ctx) ctx->err = "unknown error";
        return OFLOW_ERR_CUDA;
    }
}

// Synchronous unless the caller supplied a stream and wants device outputs.
void finish(oflow_ctx *ctx, bool device_only) {
    if (ctx->user && device_only) return;
    OF_CUDA(cudaStreamSynchronize(ctx->stream()));
}

// Side streams and events of the chunked host solves, created on first use.
void make_side_streams(oflow_ctx *ctx) {
    if (ctx->fork) return;
    for (int c = 0; c < kHostChunks; c++) {
        OF_CUDA(cudaStreamCreateWithFlags(&ctx->side[c], cudaStreamNonBlocking));
        OF_CUDA(cudaEventCreateWithFlags(&ctx->join[c], cudaEventDisableTiming));
    }
    OF_CUDA(cudaEventCreateWithFlags(&ctx->fork, cudaEventDisableTiming));
}

// The plan of chunk slot c for this size and batch (chunks run at once, so
// each slot has plans of its own).
// resident-slot share of a chunk's queue launches (OFLOW_SIDE_QUEUE=n: 1/n)
int side_share(int chunks) {
    const char *e = getenv("OFLOW_SIDE_QUEUE");
    const int n = e ? atoi(e) : 0;
    return n > 0 ? n : chunks;
}

// Chunks of a host batch (OFLOW_HOST_CHUNKS, 1..kHostChunks; default 1).
int host_chunks() {
    const char *e = getenv("OFLOW_HOST_CHUNKS");
    const int n = e ? atoi(e) : 1;
    return n < 1 ? 1 : (n > kHostChunks ? kHostChunks : n);
}

TvPlan &side_plan(oflow_ctx *ctx, int c, int chunks, int w, int h, int B, int dtype,
                  const oflow_tvl1_params &p) {
    auto &v = ctx->tv_side[c];
    for (auto &pl : v)
        if (pl->width() == w && pl->height() == h && pl->batch() == B && pl->dtype() == dtype &&
            same(pl->params(), p)) {
            pl->set_share(side_share(chunks));
            return *pl;
        }
    v.emplace_back(new TvPlan(w, h, B, dtype, p, false, &ctx->tune));
    // chunks share the GPU: one launch per block of iterations, interleaving
    // with the other chunks' kernels.  OFLOW_SIDE_QUEUE=n runs the work queue
    // instead, each chunk's launches on 1/n of the resident slots; measured
    // end to end: 1,118 pairs/s with n = 4 and 954 with n = 1, against 1,133
    // (persistent blocks hold SMs the other chunks' kernels need).
    const char *e = getenv("OFLOW_SIDE_QUEUE");
    const int sq = e ? atoi(e) : 0;
    v.back()->use_queue(sq > 0);
    v.back()->set_share(side_share(chunks));
    if (v.size() > kMaxPlans) ctx->last_tv.clear();  // an evicted plan may be listed
    keep_recent(v);
    return *v.back();
}

TvPlan &tv_plan(oflow_ctx *ctx, int w, int h, int B, int dtype, const oflow_tvl1_params &p,
                bool trace) {
    for (auto &pl : ctx->tv)
        if (pl->width() == w && pl->height() == h && pl->batch() == B && pl->dtype() == dtype &&
            pl->traced() == trace && same(pl->params(), p))
            return *pl;
    ctx->tv.emplace_back(new TvPlan(w, h, B, dtype, p, trace, &ctx->tune));
    if (ctx->tv.size() > kMaxPlans) ctx->last_tv.clear();  // an evicted plan may be listed
    keep_recent(ctx->tv);
    return *ctx->tv.back();
}

void check_tvl1_params(const oflow_tvl1_params *p) {
    OF_CHECK(p != nullptr, "tvl1: null params");
    OF_CHECK(p->nscales >= 1, "tvl1: nscales must be >= 1");
    OF_CHECK(p->tau > 0 && p->lambda >= 0 && p->theta > 0 && p->epsilon >= 0,
             "tvl1: tau, theta must be > 0 and lambda, epsilon >= 0");
}

// Groups the pairs of a batch by (w, h, dtype); each group is one plan.
struct Group {
    int w, h, dtype;
    std::vector<int> idx;
};

std::vector<Group> group_pairs(int n, const oflow_image *I0, const oflow_image *I1) {
    std::vector<Group> g;
    for (int i = 0; i < n; i++) {
        check_image(&I0[i], "I0");
        check_image(&I1[i], "I1");
        OF_CHECK(I0[i].width == I1[i].width && I0[i].height == I1[i].height,
                 "frames of a pair differ in size");
        OF_CHECK(I0[i].dtype == I1[i].dtype, "frames of a pair differ in dtype");
        auto it = std::find_if(g.begin(), g.end(), [&](const Group &x) {
            return x.w == I0[i].width && x.h == I0[i].height && x.dtype == I0[i].dtype;
        });
        if (it == g.end()) {
            g.push_back({I0[i].width, I0[i].height, I0[i].dtype, {}});
            it = g.end() - 1;
        }
        it->idx.push_back(i);
    }
    return g;
}

// Points a plan's frame and output tables at one group's pairs: device frames
// and flows are read and written in place; host frames are staged into the
// plan's buffers and host flows come from its output buffer (copied after the
// run by the caller).
template <typename Plan>
void bind_pairs(Plan &pl, const Group &g, const oflow_image *I0, const oflow_image *I1,
                const oflow_flow *out, cudaStream_t s) {
    for (size_t b = 0; b < g.idx.size(); b++) {
        const int bi = (int)b;
        const oflow_image *im[2] = {&I0[g.idx[b]], &I1[g.idx[b]]};
        for (int k = 0; k < 2; k++) {
            if (im[k]->location == OFLOW_DEVICE) {
                pl.bind_frame(bi, k, im[k]->data, im[k]->pitch);
            } else {
                stage_image(*im[k], pl.raw_input(bi, k), dtype_size(g.dtype), s);
                pl.bind_raw(bi, k);
            }
        }
        const oflow_flow &o = out[g.idx[b]];
        if (o.location == OFLOW_DEVICE)
            pl.bind_out(bi, o.u, o.v, o.pitch);
        else
            pl.bind_own_out(bi);
    }
}

void run_tvl1(oflow_ctx *ctx, int n, const oflow_image *I0, const oflow_image *I1,
              const oflow_tvl1_params *p, const oflow_flow *out, oflow_tvl1_stats *stats,
              double *energy_trace, oflow_tvl1_profile *prof = nullptr) {
    OF_CHECK(ctx != nullptr, "null context");
    OF_CHECK(n >= 1 && I0 && I1 && out, "tvl1: empty batch or null arrays");
    check_tvl1_params(p);
    for (int i = 0; i < n; i++) check_flow(&out[i], I0[i].width);
    const cudaStream_t st = ctx->stream();
    bool device_only = stats == nullptr && energy_trace == nullptr && prof == nullptr;
    const std::vector<Group> groups = group_pairs(n, I0, I1);
    OF_CHECK(prof == nullptr || groups.size() == 1, "tvl1 profile: pairs must share one size");
    ctx->last_tv.clear();
    // stages the group's pairs [b0, b1) into plan pl on stream s: device frames
    // are read in place (pitched), host frames are copied
    auto bind = [&](TvPlan &pl, const Group &g, int b0, int b1, cudaStream_t s) {
        for (int b = b0; b < b1; b++) {
            const oflow_image *im[2] = {&I0[g.idx[b]], &I1[g.idx[b]]};
            for (int k = 0; k < 2; k++) {
                if (im[k]->location == OFLOW_DEVICE) {
                    pl.bind_frame(b - b0, k, im[k]->data, im[k]->pitch ? im[k]->pitch : im[k]->width);
                } else {
                    stage_image(*im[k], pl.raw_input(b - b0, k), dtype_size(g.dtype), s);
                    pl.bind_raw(b - b0, k);
                }
            }
            // device flows are written in place by the schedule's last kernel
            const oflow_flow &o = out[g.idx[b]];
            if (o.location == OFLOW_DEVICE)
                pl.bind_out(b - b0, o.u, o.v, o.pitch);
            else
                pl.bind_own_out(b - b0);
        }
    };
    auto collect = [&](TvPlan &pl, const Group &g, int b0, int b1, cudaStream_t s) {
        if (stats) pl.compute_energy(s);
        for (int b = b0; b < b1; b++) {
            const oflow_flow &o = out[g.idx[b]];
            if (o.location == OFLOW_HOST) {
                unstage_plane(pl.out_u(b - b0), g.w, g.h, o.u, o.pitch, o.location, s);
                unstage_plane(pl.out_v(b - b0), g.w, g.h, o.v, o.pitch, o.location, s);
                device_only = false;
            }
            if (stats) pl.read_stats(b - b0, &stats[g.idx[b]], s);
        }
    };
    for (const Group &g : groups) {
        const int ng = (int)g.idx.size();
        bool host_io = false;
        for (int i : g.idx)
            host_io = host_io || I0[i].location == OFLOW_HOST || I1[i].location == OFLOW_HOST ||
                      out[i].location == OFLOW_HOST;
        const int chunks = (host_io && !prof && !energy_trace)
                               ? std::max(1, std::min(host_chunks(), ng / kChunkMinPairs))
                               : 1;
        if (chunks > 1) {
            // chunk c: pairs [c*ng/chunks, (c+1)*ng/chunks) on side stream c
            make_side_streams(ctx);
            OF_CUDA(cudaEventRecord(ctx->fork, st));
            for (int c = 0; c < chunks; c++) {
                const int b0 = c * ng / chunks, b1 = (c + 1) * ng / chunks;
                const cudaStream_t sc = ctx->side[c];
                TvPlan &pl = side_plan(ctx, c, chunks, g.w, g.h, b1 - b0, g.dtype, *p);
                ctx->last_tv.push_back(&pl);
                pl.check_device_error();  // a failure of an earlier, unsynchronised call
                OF_CUDA(cudaStreamWaitEvent(sc, ctx->fork, 0));
                bind(pl, g, b0, b1, sc);
                pl.run(sc);
                collect(pl, g, b0, b1, sc);
                OF_CUDA(cudaEventRecord(ctx->join[c], sc));
                OF_CUDA(cudaStreamWaitEvent(st, ctx->join[c], 0));
            }
            continue;
        }
        TvPlan &pl = tv_plan(ctx, g.w, g.h, ng, g.dtype, *p, energy_trace != nullptr);
        if (!prof && !energy_trace) ctx->last_tv.push_back(&pl);
        pl.check_device_error();  // a failure of an earlier, unsynchronised call
        bind(pl, g, 0, ng, st);
        if (prof)
            pl.profile(st, prof);
        else if (energy_trace)
            pl.run_eager(st);
        else
            pl.run(st);
        collect(pl, g, 0, ng, st);
        if (energy_trace) pl.read_energy_trace(0, energy_trace, st);
    }
    finish(ctx, device_only);
    for (TvPlan *pl : ctx->last_tv) pl->check_device_error();
}

}  // namespace

// Detaches the nets and streams of a context being destroyed: their handles
// stay valid for destroy calls but no longer reach the context.
static void detach_children(oflow_ctx *ctx);

extern "C" {

int oflow_abi_version(void) { return OFLOW_ABI_VERSION; }

const char *oflow_status_string(int s) {
    switch (s) {
        case OFLOW_OK: return "ok";
        case OFLOW_ERR_BAD_ARG: return "bad argument";
        case OFLOW_ERR_CUDA: return "CUDA error";
        case OFLOW_ERR_TIMEOUT: return "device wait timed out";
        case OFLOW_ERR_NO_DEVICE: return "no CUDA device";
        case OFLOW_ERR_OOM: return "out of memory";
        case OFLOW_ERR_UNSUPPORTED: return "unsupported";
        default: return "unknown status";
    }
}

oflow_status oflow_ctx_create(int device, oflow_ctx **out) {
    if (!out) return OFLOW_ERR_BAD_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return OFLOW_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= count) return OFLOW_ERR_BAD_ARG;
    oflow_ctx *ctx = new (std::nothrow) oflow_ctx();
    if (!ctx) return OFLOW_ERR_OOM;
    ctx->device = device;
    const oflow_status s = guard(ctx, [&] {
        // a blocking stream: work a caller queued on the legacy default stream
        // (e.g. torch's) is ordered before ours without extra events
        OF_CUDA(cudaStreamCreateWithFlags(&ctx->own, cudaStreamDefault));
    });
    if (s != OFLOW_OK) {
        delete ctx;
        return s;
    }
    *out = ctx;
    return OFLOW_OK;
}

oflow_status oflow_ctx_destroy(oflow_ctx *ctx) {
    if (!ctx) return OFLOW_ERR_BAD_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream());
    detach_children(ctx);
    ctx->tv.clear();
    ctx->hs.clear();
    ctx->pyrlk.clear();
    ctx->lk.clear();
    ctx->mixed.clear();
    ctx->tv_warm.clear();
    for (int c = 0; c < kHostChunks; c++) {
        if (ctx->side[c]) cudaStreamSynchronize(ctx->side[c]);
        ctx->tv_side[c].clear();
        if (ctx->side[c]) cudaStreamDestroy(ctx->side[c]);
        if (ctx->join[c]) cudaEventDestroy(ctx->join[c]);
    }
    if (ctx->fork) cudaEventDestroy(ctx->fork);
    if (ctx->own) cudaStreamDestroy(ctx->own);
    delete ctx;
    return OFLOW_OK;
}

oflow_status oflow_ctx_set_stream(oflow_ctx *ctx, void *stream) {
    if (!ctx) return OFLOW_ERR_BAD_ARG;
    ctx->user = static_cast<cudaStream_t>(stream);
    return OFLOW_OK;
}

oflow_status oflow_ctx_trim(oflow_ctx *ctx) {
    if (!ctx) return OFLOW_ERR_BAD_ARG;
    return guard(ctx, [&] {
        OF_CUDA(cudaStreamSynchronize(ctx->stream()));
        ctx->last_tv.clear();
        ctx->tv.clear();
        ctx->hs.clear();
        ctx->pyrlk.clear();
        ctx->lk.clear();
        ctx->mixed.clear();
        ctx->tv_warm.clear();
        for (auto &v : ctx->tv_side) v.clear();
    });
}

const char *oflow_ctx_last_error(const oflow_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void oflow_tvl1_default_params(oflow_tvl1_params *p) {
    if (!p) return;
    p->tau = 0.25f;
    p->lambda = 0.15f;
    p->theta = 0.3f;
    p->nscales = 100;
    p->zfactor = 0.5f;
    p->warps = 5;
    p->epsilon = 0.01f;
    p->max_iterations = 300;
}

int oflow_tvl1_nscales(int w, int h, const oflow_tvl1_params *p) {
    if (!p || w <= 0 || h <= 0 || !(p->zfactor > 0.0f && p->zfactor < 1.0f)) return -1;
    return tvl1_nscales(w, h, p->nscales, p->zfactor);
}

oflow_status oflow_tvl1(oflow_ctx *ctx, const oflow_image *I0, const oflow_image *I1,
                        const oflow_tvl1_params *p, const oflow_flow *out,
                        oflow_tvl1_stats *stats) {
    return guard(ctx, [&] { run_tvl1(ctx, 1, I0, I1, p, out, stats, nullptr); });
}

oflow_status oflow_tvl1_batch(oflow_ctx *ctx, int n, const oflow_image *I0,
                              const oflow_image *I1, const oflow_tvl1_params *p,
                              const oflow_flow *out, oflow_tvl1_stats *stats) {
    return guard(ctx, [&] { run_tvl1(ctx, n, I0, I1, p, out, stats, nullptr); });
}

oflow_status oflow_tvl1_batch_profile(oflow_ctx *ctx, int n, const oflow_image *I0,
                                      const oflow_image *I1, const oflow_tvl1_params *p,
                                      const oflow_flow *out, oflow_tvl1_stats *stats,
                                      oflow_tvl1_profile *prof) {
    return guard(ctx, [&] {
        OF_CHECK(prof != nullptr, "tvl1 profile: null profile");
        run_tvl1(ctx, n, I0, I1, p, out, stats, nullptr, prof);
    });
}

oflow_status oflow_tvl1_energy_trace(oflow_ctx *ctx, const oflow_image *I0,
                                     const oflow_image *I1, const oflow_tvl1_params *p,
                                     const oflow_flow *out, oflow_tvl1_stats *stats,
                                     double *energy) {
    return guard(ctx, [&] {
        OF_CHECK(energy != nullptr, "tvl1 trace: null energy buffer");
        run_tvl1(ctx, 1, I0, I1, p, out, stats, energy);
    });
}

oflow_status oflow_tvl1_autotune(oflow_ctx *ctx, int n, const oflow_image *I0,
                                 const oflow_image *I1, const oflow_tvl1_params *p,
                                 int *cfg_per_scale) {
    return guard(ctx, [&] {
        OF_CHECK(ctx != nullptr, "null context");
        OF_CHECK(n >= 1 && I0 && I1, "tvl1 autotune: empty batch");
        check_tvl1_params(p);
        const std::vector<Group> groups = group_pairs(n, I0, I1);
        OF_CHECK(groups.size() == 1, "tvl1 autotune: pairs must share one size");
        const Group &g = groups[0];
        const cudaStream_t st = ctx->stream();
        TvPlan &pl = tv_plan(ctx, g.w, g.h, n, g.dtype, *p, false);
        for (int b = 0; b < n; b++) stage_pair_raw(pl, b, I0[b], I1[b], st);
        pl.run(st);
        pl.autotune(st, &ctx->tune);
        OF_CUDA(cudaStreamSynchronize(st));
        pl.check_device_error();
        if (cfg_per_scale)
            for (int s = 0; s < OFLOW_MAX_SCALES; s++)
                cfg_per_scale[s] = s < pl.nscales() ? pl.tb_config(s) : -1;
    });
}

oflow_status oflow_batch(oflow_ctx *ctx, int n, const oflow_job *jobs) {
    return guard(ctx, [&] {
        OF_CHECK(ctx != nullptr && jobs != nullptr && n >= 1, "batch: empty or null");
        // group key per job
        std::vector<std::string> gkeys;
        std::vector<std::vector<int>> members;
        for (int i = 0; i < n; i++) {
            const oflow_job &j = jobs[i];
            check_image(&j.I0, "I0");
            check_image(&j.I1, "I1");
            check_flow(&j.out, j.I0.width);
            OF_CHECK(j.I0.width == j.I1.width && j.I0.height == j.I1.height && j.I0.dtype == j.I1.dtype,
                     "batch: frames of a pair differ");
            std::string k;
            char hdr[64];
            snprintf(hdr, sizeof hdr, "%d:%d:%d:%d:", j.solver, j.I0.width, j.I0.height, j.I0.dtype);
            k = hdr;
            if (j.solver == OFLOW_SOLVER_TVL1) {
                check_tvl1_params(j.tvl1);
                k.append(reinterpret_cast<const char *>(j.tvl1), sizeof(oflow_tvl1_params));
            } else if (j.solver == OFLOW_SOLVER_HS) {
                OF_CHECK(j.hs != nullptr, "batch: null hs params");
                k.append(reinterpret_cast<const char *>(j.hs), sizeof(oflow_hs_params));
            } else {
                throw Error(OFLOW_ERR_BAD_ARG, "batch: unknown solver");
            }
            auto it = std::find(gkeys.begin(), gkeys.end(), k);
            if (it == gkeys.end()) {
                gkeys.push_back(k);
                members.emplace_back();
                it = gkeys.end() - 1;
            }
            members[it - gkeys.begin()].push_back(i);
        }
        std::vector<std::string> comp;
        for (size_t g = 0; g < gkeys.size(); g++)
            comp.push_back(gkeys[g] + "#" + std::to_string(members[g].size()));
        MixedBatch *mb = nullptr;
        for (auto &m : ctx->mixed)
            if (m->key == comp) mb = m.get();
        if (!mb) {
            std::unique_ptr<MixedBatch> m(new MixedBatch());
            m->key = comp;
            m->members = members;
            for (size_t g = 0; g < gkeys.size(); g++) {
                const oflow_job &j = jobs[members[g][0]];
                const int B = (int)members[g].size();
                m->kind.push_back(j.solver);
                if (j.solver == OFLOW_SOLVER_TVL1) {
                    m->slot.push_back((int)m->tv.size());
                    m->tv.emplace_back(new TvPlan(j.I0.width, j.I0.height, B, j.I0.dtype, *j.tvl1,
                                                  false, &ctx->tune));
                    // groups run concurrently: by default one launch per block
                    // of iterations, interleaving with the other groups'
                    // kernels (OFLOW_MIXED_QUEUE=1: the work queue on a share
                    // of the SMs per TV-L1 group; measured 662 against 986
                    // pairs/s on the 256-pair mixed workload)
                    const char *e = getenv("OFLOW_MIXED_QUEUE");
                    m->tv.back()->use_queue(e && atoi(e) != 0);
                } else {
                    m->slot.push_back((int)m->hs.size());
                    m->hs.emplace_back(new HsPlan(j.I0.width, j.I0.height, B, j.I0.dtype, *j.hs,
                                                  &ctx->tune));
                }
                cudaStream_t s;
                OF_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
                m->streams.push_back(s);
                cudaEvent_t e;
                OF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
                m->events.push_back(e);
            }
            for (auto &t : m->tv) t->set_share((int)m->tv.size());
            cudaEvent_t fork;
            OF_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
            m->events.push_back(fork);
            ctx->mixed.emplace_back(std::move(m));
            while (ctx->mixed.size() > 4) ctx->mixed.erase(ctx->mixed.begin());
            mb = ctx->mixed.back().get();
        }
        const cudaStream_t st = ctx->stream();
        const size_t G = mb->kind.size();
        // device frames and flows in place through the plans' tables; host
        // ones through the plans' own buffers
        auto bind_group = [&](auto &pl, size_t g, cudaStream_t s) {
            for (size_t b = 0; b < mb->members[g].size(); b++) {
                const oflow_job &j = jobs[mb->members[g][b]];
                const oflow_image *im[2] = {&j.I0, &j.I1};
                for (int k = 0; k < 2; k++) {
                    if (im[k]->location == OFLOW_DEVICE) {
                        pl.bind_frame((int)b, k, im[k]->data, im[k]->pitch ? im[k]->pitch : im[k]->width);
                    } else {
                        stage_image(*im[k], pl.raw_input((int)b, k), dtype_size(im[k]->dtype), s);
                        pl.bind_raw((int)b, k);
                    }
                }
                if (j.out.location == OFLOW_DEVICE)
                    pl.bind_out((int)b, j.out.u, j.out.v, j.out.pitch);
                else
                    pl.bind_own_out((int)b);
            }
        };
        auto stage = [&](size_t g, cudaStream_t s) {
            if (mb->kind[g] == OFLOW_SOLVER_TVL1)
                bind_group(*mb->tv[mb->slot[g]], g, s);
            else
                bind_group(*mb->hs[mb->slot[g]], g, s);
        };
        bool device_only = true;
        auto unstage = [&](size_t g, cudaStream_t s) {
            for (size_t b = 0; b < mb->members[g].size(); b++) {
                const oflow_job &j = jobs[mb->members[g][b]];
                if (j.out.location != OFLOW_HOST) continue;  // written in place
                const float *ou = mb->kind[g] == OFLOW_SOLVER_TVL1 ? mb->tv[mb->slot[g]]->out_u((int)b)
                                                                   : mb->hs[mb->slot[g]]->out_u((int)b);
                const float *ov = mb->kind[g] == OFLOW_SOLVER_TVL1 ? mb->tv[mb->slot[g]]->out_v((int)b)
                                                                   : mb->hs[mb->slot[g]]->out_v((int)b);
                unstage_plane(ou, j.I0.width, j.I0.height, j.out.u, j.out.pitch, j.out.location, s);
                unstage_plane(ov, j.I0.width, j.I0.height, j.out.v, j.out.pitch, j.out.location, s);
                device_only = false;
            }
        };
        bool host_io = false;
        for (int i = 0; i < n; i++)
            host_io = host_io || jobs[i].I0.location == OFLOW_HOST || jobs[i].I1.location == OFLOW_HOST ||
                      jobs[i].out.location == OFLOW_HOST;
        if (host_io) {
            // each group on its own stream: its copies in and out overlap the
            // other groups' solves (each plan replays its own graph)
            cudaEvent_t fork = mb->events.back();
            OF_CUDA(cudaEventRecord(fork, st));
            for (size_t g = 0; g < G; g++) {
                const cudaStream_t sg = mb->streams[g];
                OF_CUDA(cudaStreamWaitEvent(sg, fork, 0));
                stage(g, sg);
                if (mb->kind[g] == OFLOW_SOLVER_TVL1)
                    mb->tv[mb->slot[g]]->run(sg);
                else
                    mb->hs[mb->slot[g]]->run(sg);
                unstage(g, sg);
                OF_CUDA(cudaEventRecord(mb->events[g], sg));
                OF_CUDA(cudaStreamWaitEvent(st, mb->events[g], 0));
            }
        } else {
            // device buffers: copies on the context stream, then all groups as
            // the branches of one graph
            for (size_t g = 0; g < G; g++) {
                stage(g, st);
                if (mb->kind[g] == OFLOW_SOLVER_TVL1)
                    mb->tv[mb->slot[g]]->upload_frames(st);
                else
                    mb->hs[mb->slot[g]]->upload_io(st);
            }
            if (!mb->graph.ready()) {
                mb->graph.capture(st, [&](cudaStream_t s) {
                    cudaEvent_t fork = mb->events.back();
                    OF_CUDA(cudaEventRecord(fork, s));
                    for (size_t g = 0; g < G; g++) {
                        OF_CUDA(cudaStreamWaitEvent(mb->streams[g], fork, 0));
                        if (mb->kind[g] == OFLOW_SOLVER_TVL1)
                            mb->tv[mb->slot[g]]->record(mb->streams[g]);
                        else
                            mb->hs[mb->slot[g]]->record(mb->streams[g]);
                        OF_CUDA(cudaEventRecord(mb->events[g], mb->streams[g]));
                        OF_CUDA(cudaStreamWaitEvent(s, mb->events[g], 0));
                    }
                });
            }
            mb->graph.launch(st);
            for (size_t g = 0; g < G; g++) unstage(g, st);
        }
        finish(ctx, device_only);
        for (auto &t : mb->tv) t->check_device_error();
        for (auto &t : mb->hs) t->check_device_error();
    });
}

oflow_status oflow_ctx_save_tuning(oflow_ctx *ctx, const char *path) {
    return guard(ctx, [&] {
        OF_CHECK(ctx != nullptr && path != nullptr, "save tuning: null argument");
        FILE *f = fopen(path, "w");
        OF_CHECK(f != nullptr, std::string("save tuning: cannot open ") + path);
        fprintf(f, "# oflow tuning table: solver level_width level_height batch config\n");
        for (const auto &kv : ctx->tune)
            fprintf(f, "%s %d %d %d %d\n", std::get<0>(kv.first) == kTuneHs ? "hs" : "tvl1",
                    std::get<1>(kv.first), std::get<2>(kv.first), std::get<3>(kv.first), kv.second);
        fclose(f);
    });
}

oflow_status oflow_ctx_load_tuning(oflow_ctx *ctx, const char *path) {
    return guard(ctx, [&] {
        OF_CHECK(ctx != nullptr && path != nullptr, "load tuning: null argument");
        FILE *f = fopen(path, "r");
        OF_CHECK(f != nullptr, std::string("load tuning: cannot open ") + path);
        char line[256], solver[16];
        int w, h, B, c, bad = 0;
        while (fgets(line, sizeof line, f)) {
            if (line[0] == '#' || line[0] == '\n') continue;
            if (sscanf(line, "%15s %d %d %d %d", solver, &w, &h, &B, &c) != 5 || c < 0) {
                bad = 1;
                break;
            }
            const int kind = std::string(solver) == "hs" ? kTuneHs : kTuneTvl1;
            ctx->tune[tune_key(w, h, B, kind)] = c;
        }
        fclose(f);
        OF_CHECK(!bad, "load tuning: malformed line");
        ctx->tv.clear();  // plans pick the table up when rebuilt
        for (auto &v : ctx->tv_side) v.clear();
        ctx->last_tv.clear();
        ctx->hs.clear();
    });
}

void oflow_hs_default_params(oflow_hs_params *p) {
    if (!p) return;
    p->alpha = 0.2f;
    p->nlevels = 5;
    p->nwarp = 3;
    p->nsolver = 150;
}

// cached Horn-Schunck plan of this size, batch, dtype and parameters
static HsPlan &hs_plan(oflow_ctx *ctx, int w, int h, int B, int dtype, const oflow_hs_params &p) {
    for (auto &q : ctx->hs)
        if (q->width() == w && q->height() == h && q->batch() == B && q->dtype() == dtype &&
            same(q->params(), p))
            return *q;
    ctx->hs.emplace_back(new HsPlan(w, h, B, dtype, p, &ctx->tune));
    HsPlan *pl = ctx->hs.back().get();
    keep_recent(ctx->hs);
    return *pl;
}

oflow_status oflow_hs_batch(oflow_ctx *ctx, int n, const oflow_image *I0,
                            const oflow_image *I1, const oflow_hs_params *p,
                            const oflow_flow *out) {
    return guard(ctx, [&] {
        OF_CHECK(ctx != nullptr, "null context");
        OF_CHECK(n >= 1 && I0 && I1 && out && p, "hs: empty batch or null arrays");
        for (int i = 0; i < n; i++) check_flow(&out[i], I0[i].width);
        const cudaStream_t st = ctx->stream();
        bool device_only = true;
        std::vector<HsPlan *> ran;
        for (const Group &g : group_pairs(n, I0, I1)) {
            HsPlan *pl = &hs_plan(ctx, g.w, g.h, (int)g.idx.size(), g.dtype, *p);
            ran.push_back(pl);
            bind_pairs(*pl, g, I0, I1, out, st);
            pl->run(st);
            for (size_t b = 0; b < g.idx.size(); b++) {
                const oflow_flow &o = out[g.idx[b]];
                if (o.location != OFLOW_HOST) continue;  // written in place
                unstage_plane(pl->out_u((int)b), g.w, g.h, o.u, o.pitch, o.location, st);
                unstage_plane(pl->out_v((int)b), g.w, g.h, o.v, o.pitch, o.location, st);
                device_only = false;
            }
        }
        finish(ctx, device_only);
        for (HsPlan *pl : ran) pl->check_device_error();
    });
}

oflow_status oflow_hs(oflow_ctx *ctx, const oflow_image *I0, const oflow_image *I1,
                      const oflow_hs_params *p, const oflow_flow *out) {
    return oflow_hs_batch(ctx, 1, I0, I1, p, out);
}

oflow_status oflow_hs_autotune(oflow_ctx *ctx, int n, const oflow_image *I0,
                               const oflow_image *I1, const oflow_hs_params *p,
                               int *cfg_per_level) {
    return guard(ctx, [&] {
        OF_CHECK(ctx != nullptr, "null context");
        OF_CHECK(n >= 1 && I0 && I1 && p, "hs autotune: empty batch or null arrays");
        const std::vector<Group> groups = group_pairs(n, I0, I1);
        OF_CHECK(groups.size() == 1, "hs autotune: pairs must share one size");
        const Group &g = groups[0];
        const cudaStream_t st = ctx->stream();
        HsPlan &pl = hs_plan(ctx, g.w, g.h, n, g.dtype, *p);
        for (int b = 0; b < n; b++) {
            stage_image(I0[g.idx[b]], pl.raw_input(b, 0), dtype_size(g.dtype), st);
            stage_image(I1[g.idx[b]], pl.raw_input(b, 1), dtype_size(g.dtype), st);
            pl.bind_raw(b, 0);
            pl.bind_raw(b, 1);
            pl.bind_own_out(b);
        }
        pl.run(st);
        pl.autotune(st, &ctx->tune);
        OF_CUDA(cudaStreamSynchronize(st));
        if (cfg_per_level)
            for (int l = 0; l < OFLOW_MAX_SCALES; l++)
                cfg_per_level[l] = l < pl.levels() ? pl.jacobi_config(l) : -1;
    });
}

void oflow_lk_default_params(oflow_lk_params *p) {
    if (!p) return;
    p->spac = 3;
    p->temp = 2;
    p->window = 5;
    p->levels = 3;
    p->iters = 3;
}

oflow_status oflow_lk(oflow_ctx *ctx, const oflow_image *frames, int iframe,
                      const oflow_lk_params *p, const oflow_flow *out) {
    return guard(ctx, [&] {
        OF_CHECK(ctx != nullptr && frames != nullptr && p != nullptr, "lk: null argument");
        OF_CHECK(iframe >= 0, "lk: iframe < 0");
        const int T = p->temp;
        OF_CHECK(T >= 1 && T <= 9, "lk: temporal filter size out of range");
        for (int k = 0; k < T; k++) {
            check_image(&frames[k], "frame");
            OF_CHECK(frames[k].dtype == OFLOW_U8, "lk: ring frames must be uint8");
            OF_CHECK(frames[k].width == frames[0].width && frames[k].height == frames[0].height,
                     "lk: ring frames differ in size");
        }
        const int w = frames[0].width, h = frames[0].height;
        check_flow(out, w);
        LkPlan *pl = nullptr;
        for (auto &q : ctx->lk)
            if (q->width() == w && q->height() == h && same(q->params(), *p)) pl = q.get();
        if (!pl) {
            ctx->lk.emplace_back(new LkPlan(w, h, *p));
            keep_recent(ctx->lk);
            pl = ctx->lk.back().get();
        }
        const cudaStream_t st = ctx->stream();
        for (int k = 0; k < T; k++) stage_image(frames[k], pl->ring_slot(k), 1, st);
        pl->run(iframe, st);
        unstage_plane(pl->out_u(), w, h, out->u, out->pitch, out->location, st);
        unstage_plane(pl->out_v(), w, h, out->v, out->pitch, out->location, st);
        finish(ctx, out->location == OFLOW_DEVICE);
    });
}

oflow_status oflow_pyrlk_batch(oflow_ctx *ctx, int n, const oflow_image *I0,
                               const oflow_image *I1, const oflow_lk_params *p,
                               const oflow_flow *out) {
    return guard(ctx, [&] {
        OF_CHECK(ctx != nullptr && p != nullptr, "pyrlk: null argument");
        OF_CHECK(n >= 1 && I0 && I1 && out, "pyrlk: empty batch or null arrays");
        OF_CHECK(p->temp == 2, "pyrlk: temporal filter must be the 2-tap difference");
        for (int i = 0; i < n; i++) check_flow(&out[i], I0[i].width);
        const cudaStream_t st = ctx->stream();
        bool device_only = true;
        for (const Group &g : group_pairs(n, I0, I1)) {
            const int B = (int)g.idx.size();
            PyrLkPlan *pl = nullptr;
            for (auto &q : ctx->pyrlk)
                if (q->width() == g.w && q->height() == g.h && q->batch() == B &&
                    q->dtype() == g.dtype && same(q->params(), *p))
                    pl = q.get();
            if (!pl) {
                ctx->pyrlk.emplace_back(new PyrLkPlan(g.w, g.h, B, g.dtype, *p));
                keep_recent(ctx->pyrlk);
                pl = ctx->pyrlk.back().get();
            }
            bind_pairs(*pl, g, I0, I1, out, st);
            pl->run(st);
            for (int b = 0; b < B; b++) {
                const oflow_flow &o = out[g.idx[b]];
                if (o.location != OFLOW_HOST) continue;  // written in place
                unstage_plane(pl->out_u(b), g.w, g.h, o.u, o.pitch, o.location, st);
                unstage_plane(pl->out_v(b), g.w, g.h, o.v, o.pitch, o.location, st);
                device_only = false;
            }
        }
        finish(ctx, device_only);
    });
}

oflow_status oflow_pyrlk(oflow_ctx *ctx, const oflow_image *I0, const oflow_image *I1,
                         const oflow_lk_params *p, const oflow_flow *out) {
    return oflow_pyrlk_batch(ctx, 1, I0, I1, p, out);
}

}  // extern "C"

struct oflow_net {
    oflow_ctx *ctx;
    std::unique_ptr<WarmNet> net;
};

extern "C" {

int oflow_net_num_params(void) { return warmnet_num_params(); }

oflow_status oflow_net_create(oflow_ctx *ctx, int width, int height, int batch, oflow_net **out) {
    if (!out) return OFLOW_ERR_BAD_ARG;
    *out = nullptr;
    return guard(ctx, [&] {
        OF_CHECK(ctx != nullptr, "null context");
        std::unique_ptr<oflow_net> n(new oflow_net());
        n->ctx = ctx;
        n->net.reset(new WarmNet(width, height, batch));
        ctx->nets.push_back(n.get());
        *out = n.release();
    });
}

oflow_status oflow_net_destroy(oflow_net *net) {
    if (!net) return OFLOW_ERR_BAD_ARG;
    if (net->ctx) {  // null once its context was destroyed
        cudaStreamSynchronize(net->ctx->stream());
        auto &v = net->ctx->nets;
        v.erase(std::remove(v.begin(), v.end(), net), v.end());
    }
    delete net;
    return OFLOW_OK;
}

oflow_status oflow_net_out_size(const oflow_net *net, int *w, int *h) {
    if (!net || !w || !h) return OFLOW_ERR_BAD_ARG;
    *w = net->net->out_w();
    *h = net->net->out_h();
    return OFLOW_OK;
}

oflow_status oflow_net_set_params(oflow_net *net, const float *params) {
    if (!net || !net->ctx || !params) return OFLOW_ERR_BAD_ARG;
    return guard(net->ctx, [&] { net->net->set_params(params, net->ctx->stream()); });
}

oflow_status oflow_net_get_params(oflow_net *net, float *params) {
    if (!net || !net->ctx || !params) return OFLOW_ERR_BAD_ARG;
    return guard(net->ctx, [&] { net->net->get_params(params, net->ctx->stream()); });
}

oflow_status oflow_net_train_step(oflow_net *net, const void *frames, int dtype,
                                  const float *target, float lr, double *loss) {
    if (!net || !net->ctx || !frames || !target) return OFLOW_ERR_BAD_ARG;
    return guard(net->ctx, [&] {
        OF_CHECK(dtype == OFLOW_U8 || dtype == OFLOW_F32, "net: bad dtype");
        const size_t ps = (size_t)net->net->width() * net->net->height();
        const double l = net->net->train_step(frames, dtype, ps, target, lr, net->ctx->stream());
        if (loss) *loss = l;
    });
}

oflow_status oflow_net_predict(oflow_net *net, const void *frames, int dtype, float *flow) {
    if (!net || !net->ctx || !frames || !flow) return OFLOW_ERR_BAD_ARG;
    return guard(net->ctx, [&] {
        OF_CHECK(dtype == OFLOW_U8 || dtype == OFLOW_F32, "net: bad dtype");
        const cudaStream_t st = net->ctx->stream();
        const size_t ps = (size_t)net->net->width() * net->net->height();
        net->net->forward(frames, dtype, ps, st);
        net->net->flow_to(nullptr, 0, flow, st);
        OF_CUDA(cudaGetLastError());
    });
}

oflow_status oflow_tvl1_warm(oflow_ctx *ctx, oflow_net *net, int n, const oflow_image *I0,
                             const oflow_image *I1, const oflow_tvl1_params *warm,
                             const int *warps_per_scale, const int *iters_per_scale,
                             const oflow_tvl1_params *plain, const oflow_flow *out,
                             double *energy_warm, double *energy_plain, double *epe_vs_plain,
                             int *accepted, oflow_tvl1_stats *stats) {
    return guard(ctx, [&] {
        OF_CHECK(ctx != nullptr && net != nullptr && I0 && I1 && out, "tvl1 warm: null argument");
        OF_CHECK(net->ctx != nullptr, "tvl1 warm: the network's context was destroyed");
        OF_CHECK(n == net->net->batch(), "tvl1 warm: n must equal the network batch");
        check_tvl1_params(warm);
        if (plain) check_tvl1_params(plain);
        const std::vector<Group> groups = group_pairs(n, I0, I1);
        OF_CHECK(groups.size() == 1, "tvl1 warm: pairs must share one size and dtype");
        const Group &g = groups[0];
        OF_CHECK(g.w == net->net->width() && g.h == net->net->height(),
                 "tvl1 warm: frame size differs from the network's");
        for (int i = 0; i < n; i++) check_flow(&out[i], g.w);
        const cudaStream_t st = ctx->stream();
        TvPlan *wp = nullptr;
        for (auto &q : ctx->tv_warm)
            if (q->width() == g.w && q->height() == g.h && q->batch() == n && q->dtype() == g.dtype &&
                same(q->params(), *warm) && q->same_schedule(warps_per_scale, iters_per_scale))
                wp = q.get();
        if (!wp) {
            std::unique_ptr<TvPlan> np(new TvPlan(g.w, g.h, n, g.dtype, *warm, false, &ctx->tune, 3));
            np->set_schedule(warps_per_scale, iters_per_scale);
            ctx->tv_warm.emplace_back(std::move(np));
            keep_recent(ctx->tv_warm);
            wp = ctx->tv_warm.back().get();
        }
        OF_CHECK(wp->level_w(3) == net->net->out_w() && wp->level_h(3) == net->net->out_h(),
                 "tvl1 warm: scale 3 does not match the network output");
        // the judge reads both solves' flows from the plans' own buffers
        for (int b = 0; b < n; b++) stage_pair_raw(*wp, b, I0[b], I1[b], st);
        net->net->forward(wp->raw_input(0, 0), g.dtype, wp->plane_stride(), st);
        net->net->flow_to(wp->uz(), wp->plane_stride(), nullptr, st);
        wp->run(st);
        std::vector<double> ew(n), ep(n, 0.0), er(n, 0.0);
        std::vector<int> acc(n, 1);
        wp->true_energy(ew.data(), st);  // synchronises
        wp->check_device_error();
        if (stats) {
            wp->compute_energy(st);
            for (int b = 0; b < n; b++) wp->read_stats(b, &stats[b], st);
        }
        TvPlan *pp = nullptr;
        if (plain) {
            pp = &tv_plan(ctx, g.w, g.h, n, g.dtype, *plain, false);
            for (int b = 0; b < n; b++) stage_pair_raw(*pp, b, I0[b], I1[b], st);
            pp->run(st);
            pp->true_energy(ep.data(), st);
            pp->check_device_error();
            wp->rel_epe_against(*pp, er.data(), st);
            // both within 1 %: energy, and the end-point difference from the
            // plain flow relative to the plain flow's magnitude
            for (int b = 0; b < n; b++) acc[b] = (ew[b] <= 1.01 * ep[b] && er[b] <= 0.01) ? 1 : 0;
        }
        for (int b = 0; b < n; b++) {
            const TvPlan *src = acc[b] ? wp : pp;
            unstage_plane(src->out_u(b), g.w, g.h, out[b].u, out[b].pitch, out[b].location, st);
            unstage_plane(src->out_v(b), g.w, g.h, out[b].v, out[b].pitch, out[b].location, st);
            if (energy_warm) energy_warm[b] = ew[b];
            if (energy_plain) energy_plain[b] = ep[b];
            if (epe_vs_plain) epe_vs_plain[b] = er[b];
            if (accepted) accepted[b] = acc[b];
        }
    });
}

}  // extern "C"

// A frame stream: frame k of every lane goes to slot k % 3.  A TV-L1 solve
// reads its two frames from the slots through the plan's frame table; an HS
// solve copies them into its staging buffers.  Slot k % 3 last held frame
// k - 3, read by the solves of pushes k - 3 and k - 2, so the upload of frame
// k waits for the end of solve k - 2 only and overlaps solve k - 1.
struct oflow_stream {
    oflow_ctx *ctx = nullptr;
    oflow_stream_desc desc{};
    std::unique_ptr<TvPlan> tv;
    std::unique_ptr<HsPlan> hs;
    DevBuf slots;  // [3][lanes][w*h] frames of the dtype; slot 2 starts as zeros
    long long frames = 0;
    cudaStream_t copy = nullptr;
    cudaEvent_t uploaded = nullptr;
    cudaEvent_t done[3] = {nullptr, nullptr, nullptr};
    size_t frame_bytes() const { return (size_t)desc.width * desc.height * dtype_size(desc.dtype); }
    char *slot(long long k, int lane) const {
        return slots.as<char>() + ((size_t)(k % 3) * desc.lanes + lane) * frame_bytes();
    }
    ~oflow_stream() {
        if (copy) cudaStreamDestroy(copy);
        if (uploaded) cudaEventDestroy(uploaded);
        for (cudaEvent_t e : done)
            if (e) cudaEventDestroy(e);
    }
};

extern "C" {

oflow_status oflow_stream_create(oflow_ctx *ctx, const oflow_stream_desc *desc, oflow_stream **out) {
    if (!out) return OFLOW_ERR_BAD_ARG;
    *out = nullptr;
    std::unique_ptr<oflow_stream> s;
    const oflow_status st = guard(ctx, [&] {
        OF_CHECK(ctx != nullptr && desc != nullptr, "stream: null argument");
        OF_CHECK(desc->solver == OFLOW_SOLVER_TVL1 || desc->solver == OFLOW_SOLVER_HS, "stream: bad solver");
        OF_CHECK(desc->width > 0 && desc->height > 0 && desc->lanes >= 1, "stream: bad size");
        OF_CHECK(desc->dtype == OFLOW_U8 || desc->dtype == OFLOW_F32, "stream: bad dtype");
        s.reset(new oflow_stream());
        s->ctx = ctx;
        s->desc = *desc;
        if (desc->solver == OFLOW_SOLVER_TVL1) {
            check_tvl1_params(&desc->tvl1);
            s->tv.reset(new TvPlan(desc->width, desc->height, desc->lanes, desc->dtype, desc->tvl1, false,
                                   &ctx->tune));
        } else {
            s->hs.reset(new HsPlan(desc->width, desc->height, desc->lanes, desc->dtype, desc->hs,
                                   &ctx->tune));
        }
        s->slots.alloc(3 * (size_t)desc->lanes * s->frame_bytes());
        OF_CUDA(cudaMemset(s->slots.as<char>(), 0, s->slots.bytes()));
        OF_CUDA(cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking));
        OF_CUDA(cudaEventCreateWithFlags(&s->uploaded, cudaEventDisableTiming));
        for (cudaEvent_t &e : s->done) OF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    });
    if (st == OFLOW_OK) {
        ctx->streams.push_back(s.get());
        *out = s.release();
    }
    return st;
}

oflow_status oflow_stream_destroy(oflow_stream *s) {
    if (!s) return OFLOW_OK;
    oflow_status st = OFLOW_OK;
    if (s->ctx) {  // null once its context was destroyed
        st = guard(s->ctx, [&] {
            OF_CUDA(cudaStreamSynchronize(s->copy));
            OF_CUDA(cudaStreamSynchronize(s->ctx->stream()));
        });
        auto &v = s->ctx->streams;
        v.erase(std::remove(v.begin(), v.end(), s), v.end());
    }
    delete s;
    return st;
}

long long oflow_stream_frames(const oflow_stream *s) { return s ? s->frames : -1; }

oflow_status oflow_stream_push(oflow_stream *s, const oflow_image *frames, const oflow_flow *out,
                               oflow_tvl1_stats *stats) {
    if (!s || !s->ctx) return OFLOW_ERR_BAD_ARG;
    return guard(s->ctx, [&] {
        const oflow_stream_desc &d = s->desc;
        OF_CHECK(frames != nullptr && out != nullptr, "stream: null arrays");
        for (int i = 0; i < d.lanes; i++) {
            check_image(&frames[i], "frame");
            OF_CHECK(frames[i].width == d.width && frames[i].height == d.height && frames[i].dtype == d.dtype,
                     "stream: frame differs from the stream's size or dtype");
            check_flow(&out[i], d.width);
        }
        const cudaStream_t st = s->ctx->stream();
        const long long k = s->frames;  // this push's frame index; the previous is k - 1
        if (k >= 2) OF_CUDA(cudaStreamWaitEvent(s->copy, s->done[(k - 2) % 3], 0));
        // a device frame may come from work queued on the solve stream: order
        // its copy after that (host frames are ready when push is called)
        bool any_device = false;
        for (int i = 0; i < d.lanes; i++) any_device |= frames[i].location == OFLOW_DEVICE;
        if (any_device) {
            OF_CUDA(cudaEventRecord(s->uploaded, st));
            OF_CUDA(cudaStreamWaitEvent(s->copy, s->uploaded, 0));
        }
        const size_t esz = dtype_size(d.dtype);
        for (int i = 0; i < d.lanes; i++) stage_image(frames[i], s->slot(k, i), esz, s->copy);
        OF_CUDA(cudaEventRecord(s->uploaded, s->copy));
        OF_CUDA(cudaStreamWaitEvent(st, s->uploaded, 0));
        const long long kp = k + 2;  // slot of frame k - 1 (slot 2 holds zeros before frame 2)
        for (int i = 0; i < d.lanes; i++) {
            if (s->tv) {
                s->tv->bind_frame(i, 0, s->slot(kp, i), d.width);
                s->tv->bind_frame(i, 1, s->slot(k, i), d.width);
            } else {
                OF_CUDA(cudaMemcpyAsync(s->hs->raw_input(i, 0), s->slot(kp, i), s->frame_bytes(),
                                        cudaMemcpyDeviceToDevice, st));
                OF_CUDA(cudaMemcpyAsync(s->hs->raw_input(i, 1), s->slot(k, i), s->frame_bytes(),
                                        cudaMemcpyDeviceToDevice, st));
            }
        }
        bool device_only = stats == nullptr;
        if (s->tv)
            s->tv->run(st);
        else
            s->hs->run(st);
        OF_CUDA(cudaEventRecord(s->done[k % 3], st));
        if (stats && s->tv) s->tv->compute_energy(st);
        for (int i = 0; i < d.lanes; i++) {
            const float *ou = s->tv ? s->tv->out_u(i) : s->hs->out_u(i);
            const float *ov = s->tv ? s->tv->out_v(i) : s->hs->out_v(i);
            unstage_plane(ou, d.width, d.height, out[i].u, out[i].pitch, out[i].location, st);
            unstage_plane(ov, d.width, d.height, out[i].v, out[i].pitch, out[i].location, st);
            if (out[i].location == OFLOW_HOST) device_only = false;
            if (stats && s->tv) s->tv->read_stats(i, &stats[i], st);
        }
        s->frames++;
        finish(s->ctx, device_only);
        if (s->tv) s->tv->check_device_error();
        if (s->hs) s->hs->check_device_error();
    });
}

oflow_status oflow_ctx_last_launches(oflow_ctx *ctx, long long *launches) {
    return guard(ctx, [&] {
        OF_CHECK(ctx != nullptr && launches != nullptr, "last_launches: null argument");
        long long total = 0;
        for (TvPlan *pl : ctx->last_tv) total += pl->device_launches(ctx->stream());
        *launches = total;
    });
}

oflow_status oflow_flow_to_color(oflow_ctx *ctx, int n, int width, int height,
                                 const oflow_flow *flows, const oflow_bgr_image *out) {
    return guard(ctx, [&] {
        OF_CHECK(ctx != nullptr && n >= 0 && (n == 0 || (flows && out)), "flow_to_color: null argument");
        OF_CHECK(width > 0 && height > 0, "flow_to_color: empty image");
        for (int i = 0; i < n; i++) {
            check_flow(&flows[i], width);
            OF_CHECK(out[i].data != nullptr, "flow_to_color: null output");
            OF_CHECK(out[i].location == OFLOW_HOST || out[i].location == OFLOW_DEVICE,
                     "flow_to_color: bad output location");
            OF_CHECK(out[i].pitch == 0 || out[i].pitch >= 3 * width, "flow_to_color: pitch < 3 * width");
        }
        const cudaStream_t st = ctx->stream();
        const size_t plane = (size_t)width * height * 4, img = (size_t)width * height * 3;
        bool host_side = false;
        for (int s0 = 0; s0 < n; s0 += kColorMaxJobs) {
            const int k = std::min(kColorMaxJobs, n - s0);
            // scratch: staged u, v planes and images for host-side jobs of this chunk
            size_t need = 0;
            for (int i = 0; i < k; i++) {
                if (flows[s0 + i].location == OFLOW_HOST) need += 2 * ((plane + 255) & ~size_t(255));
                if (out[s0 + i].location == OFLOW_HOST) need += (img + 255) & ~size_t(255);
            }
            if (need > ctx->color_scratch.bytes()) {
                OF_CUDA(cudaStreamSynchronize(st));  // earlier chunks may still use it
                ctx->color_scratch.alloc(need);
            }
            char *sp = ctx->color_scratch.as<char>();
            ColorJobs jobs{};
            jobs.w = width;
            jobs.h = height;
            for (int i = 0; i < k; i++) {
                const oflow_flow &f = flows[s0 + i];
                const oflow_bgr_image &o = out[s0 + i];
                ColorJob &j = jobs.j[i];
                if (f.location == OFLOW_HOST) {
                    float *du = reinterpret_cast<float *>(sp);
                    sp += (plane + 255) & ~size_t(255);
                    float *dv = reinterpret_cast<float *>(sp);
                    sp += (plane + 255) & ~size_t(255);
                    const size_t fp = (size_t)(f.pitch ? f.pitch : width) * 4;
                    OF_CUDA(cudaMemcpy2DAsync(du, (size_t)width * 4, f.u, fp, (size_t)width * 4, height,
                                              cudaMemcpyHostToDevice, st));
                    OF_CUDA(cudaMemcpy2DAsync(dv, (size_t)width * 4, f.v, fp, (size_t)width * 4, height,
                                              cudaMemcpyHostToDevice, st));
                    j.u = du;
                    j.v = dv;
                    j.fpitch = width;
                    host_side = true;
                } else {
                    j.u = f.u;
                    j.v = f.v;
                    j.fpitch = f.pitch ? f.pitch : width;
                }
                if (o.location == OFLOW_HOST) {
                    j.bgr = reinterpret_cast<uint8_t *>(sp);
                    sp += (img + 255) & ~size_t(255);
                    j.bpitch = 3 * width;
                    host_side = true;
                } else {
                    j.bgr = o.data;
                    j.bpitch = o.pitch ? o.pitch : 3 * width;
                }
            }
            launch_flow_to_color(jobs, k, st);
            OF_CUDA(cudaGetLastError());
            for (int i = 0; i < k; i++) {
                const oflow_bgr_image &o = out[s0 + i];
                if (o.location != OFLOW_HOST) continue;
                OF_CUDA(cudaMemcpy2DAsync(o.data, o.pitch ? o.pitch : 3 * width, jobs.j[i].bgr,
                                          (size_t)3 * width, (size_t)3 * width, height,
                                          cudaMemcpyDeviceToHost, st));
            }
        }
        if (host_side || !ctx->user) OF_CUDA(cudaStreamSynchronize(st));
    });
}

oflow_status oflow_conv3x3(int mode, int N, int H, int W, int C, int K, int stride, int relu,
                           int out_f32, const void *a, const void *y_act, const void *b, void *out,
                           const float *bias, float *gbias, void *stream) {
    return guard(nullptr, [&] {
        OF_CHECK(N >= 1 && H >= 1 && W >= 1 && C >= 1 && K >= 1 && (stride == 1 || stride == 2),
                 "conv3x3: bad shape");
        OF_CHECK(a && b && out, "conv3x3: null buffer");
        const ConvDims d{N, H, W, C, conv_out(H, stride), conv_out(W, stride), K, stride};
        const cudaStream_t st = static_cast<cudaStream_t>(stream);
        if (mode == 0) {
            // the tcgen05 kernel; the shape must be one it takes
            OF_CHECK(bias != nullptr, "conv3x3: null bias");
            DevBuf err(sizeof(int));
            OF_CUDA(cudaMemsetAsync(err.as<int>(), 0, sizeof(int), st));
            OF_CHECK(conv_forward_umma(d, static_cast<const __nv_bfloat16 *>(a),
                                       static_cast<const __nv_bfloat16 *>(b), bias, out, out_f32 != 0,
                                       relu != 0, err.as<int>(), st),
                     "conv3x3: shape outside the tensor-core kernel (C % 16 == 0, K % 8 == 0, K <= 128)");
            int e = 0;
            OF_CUDA(cudaMemcpyAsync(&e, err.as<int>(), sizeof(int), cudaMemcpyDeviceToHost, st));
            OF_CUDA(cudaStreamSynchronize(st));
            if (e) throw Error(OFLOW_ERR_TIMEOUT, "conv3x3: a bounded wait gave up");
        } else if (mode == 3) {
            // the mma.sync forward kernel (used by training's backward products)
            OF_CHECK(bias != nullptr, "conv3x3: null bias");
            conv_forward(d, static_cast<const __nv_bfloat16 *>(a), static_cast<const __nv_bfloat16 *>(b),
                         bias, out, out_f32 != 0, relu != 0, st);
        } else if (mode == 1) {
            // the tcgen05 kernel; the shape must be one it takes
            DevBuf err(sizeof(int)), scratch(conv_backward_data_umma_scratch(d));
            OF_CUDA(cudaMemsetAsync(err.as<int>(), 0, sizeof(int), st));
            OF_CHECK(conv_backward_data_umma(d, static_cast<const float *>(a),
                                             static_cast<const __nv_bfloat16 *>(y_act),
                                             static_cast<const __nv_bfloat16 *>(b),
                                             static_cast<float *>(out), false, scratch.as<void>(),
                                             err.as<int>(), st),
                     "conv3x3: shape outside the tensor-core kernel (C % 16 == 0, K % 8 == 0)");
            int e = 0;
            OF_CUDA(cudaMemcpyAsync(&e, err.as<int>(), sizeof(int), cudaMemcpyDeviceToHost, st));
            OF_CUDA(cudaStreamSynchronize(st));
            if (e) throw Error(OFLOW_ERR_TIMEOUT, "conv3x3: a bounded wait gave up");
        } else if (mode == 4) {
            // the mma.sync backward-data kernel
            conv_backward_data(d, static_cast<const float *>(a), static_cast<const __nv_bfloat16 *>(y_act),
                               static_cast<const __nv_bfloat16 *>(b), static_cast<float *>(out), false, st);
        } else if (mode == 2) {
            // the tcgen05 kernel; the shape must be one it takes
            OF_CHECK(gbias != nullptr, "conv3x3: null bias gradient");
            DevBuf err(sizeof(int)), scratch(conv_backward_data_umma_scratch(d));
            OF_CUDA(cudaMemsetAsync(err.as<int>(), 0, sizeof(int), st));
            OF_CHECK(conv_backward_weight_umma(d, static_cast<const float *>(a),
                                               static_cast<const __nv_bfloat16 *>(y_act),
                                               static_cast<const __nv_bfloat16 *>(b),
                                               static_cast<float *>(out), gbias, scratch.as<void>(),
                                               err.as<int>(), st),
                     "conv3x3: shape outside the tensor-core kernel (C % 16 == 0, K % 8 == 0, K <= 128)");
            int e = 0;
            OF_CUDA(cudaMemcpyAsync(&e, err.as<int>(), sizeof(int), cudaMemcpyDeviceToHost, st));
            OF_CUDA(cudaStreamSynchronize(st));
            if (e) throw Error(OFLOW_ERR_TIMEOUT, "conv3x3: a bounded wait gave up");
        } else if (mode == 5) {
            // the mma.sync backward-weight kernel
            OF_CHECK(gbias != nullptr, "conv3x3: null bias gradient");
            conv_backward_weight(d, static_cast<const float *>(a),
                                 static_cast<const __nv_bfloat16 *>(y_act),
                                 static_cast<const __nv_bfloat16 *>(b), static_cast<float *>(out), gbias, st);
        } else {
            throw Error(OFLOW_ERR_BAD_ARG, "conv3x3: bad mode");
        }
        OF_CUDA(cudaGetLastError());
    });
}

}  // extern "C"

static void detach_children(oflow_ctx *ctx) {
    for (oflow_net *n : ctx->nets) n->ctx = nullptr;
    for (oflow_stream *st : ctx->streams) {
        cudaStreamSynchronize(st->copy);
        st->ctx = nullptr;
    }
    ctx->nets.clear();
    ctx->streams.clear();
}
