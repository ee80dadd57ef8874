// TV-L1 (Zach-Pock-Bischof duality TV-L1) on B200: kernels and the batched
// plan.  Follows src/tvl1/sequential/tvl1.cpp and its helpers (mask/, zoom/,
// bicubic_interpolation/) operation for operation; the arithmetic contract is
// in common.cuh (no FMA, IEEE division, double where the reference uses double
// literals).
//
// Data layout in HBM (per pair b of a plan of B equal-size pairs, N0 = w*h):
//   raw[b][2]      staged input frames (u8 or f32)
//   T[b][2]        float scratch planes (ingest output, blur output)
//   pyr_s[b][2]    pyramid level s of I0 / I1, dense nx_s*ny_s
//   cc*[b], dv*[b] column coefficients of the warp's bicubic samples of
//                  (I1, I1x, I1y) at the current level (WarpCoef, 72 B/px)
//   WR[b]          float4 (I1wx, I1wy, rho_c, |grad I1w|^2) of the current warp
//   U[k][b]        float2 (u1, u2), k = 0..7; Uz[b] upsampled flow
//   P[k][b]        float4 (p11, p12, p21, p22), k = 0..7
// State buffers 0/1 alternate as the accepted state; 2-4 and 5-7 are two sets
// of snapshots of the blocked kernel.  Level planes are packed at the start of
// their level-0-sized buffers.
//
// Control: one TvCtrl per pair on the device.  The blocked inner-iteration
// kernel runs up to 4 iterations per launch; its last block to finish reduces
// the squared change of each iteration in a fixed order, picks the state of the
// stopping iteration (tvl1.cpp:216) and sets `stop`, after which later launches
// of that warp return at once.  The host never synchronises inside a solve, so
// the whole schedule is captured into one CUDA graph.
#include "common.cuh"
#include "internal.hpp"
#include "ptx.cuh"
#include "tvl1.hpp"

#include <cooperative_groups.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstring>

namespace oflow {

// ---------------------------------------------------------------- constants
constexpr int kIterTW = 32, kIterTH = 8, kIterNT = 256;
// blocked inner iterations: iterations per launch (= halo) and the tile
// configurations, largest first (tile TW x TH, threads); shared memory is
// 40 B per region pixel (p 16, (I1wx, I1wy, rho_c, |grad I1w|^2) 16, u 8)
constexpr int kTbK = 4;
// Inner-iteration configurations of k_tvl1_tb: tile tw x th, nt threads.
struct TbCfg {
    int tw, th, nt;
};
constexpr TbCfg kTbCfgs[] = {{64, 32, 512}, {64, 16, 256}, {32, 16, 256}, {16, 8, 128}};
constexpr int kTbNumCfgs = 4;
// Configuration 4: the whole level of a pair in one block (k_tvl1_level), for
// levels of at most kLvMaxPx pixels.
constexpr int kLevelCfg = 4;
// Configuration 5: the whole level of a pair in row bands over a cluster of
// kClC blocks (k_tvl1_cluster), for levels whose band fits shared memory.
constexpr int kClusterCfg = 5;
constexpr int kNumIterCfgs = 6;
// tile of a tiled configuration (false for the whole-level ones)
inline bool cfg_tile(int c, int &tw, int &th) {
    if (c >= 0 && c < kTbNumCfgs) {
        tw = kTbCfgs[c].tw;
        th = kTbCfgs[c].th;
        return true;
    }
    return false;
}
constexpr int kClC = 8;
constexpr size_t kClMaxSmem = 200 * 1024;
__host__ __device__ inline int cl_band_rows(int ny) { return (ny + kClC - 1) / kClC; }
// u (8 B), p (16 B) and the warp data (16 B) of a band in shared memory
inline bool cluster_fits(int nx, int ny) {
    return ny >= 2 * kClC && (size_t)cl_band_rows(ny) * nx * 40 <= kClMaxSmem;
}
constexpr int kLvNT = 1024;
constexpr int kLvMaxPx = 9216;  // u (8 B) + p (16 B) per pixel: 221,184 B of shared memory
inline bool level_fits(int nx, int ny) { return (long long)nx * ny <= kLvMaxPx; }
constexpr size_t tb_smem_bytes(int tw, int th) { return (size_t)(tw + 2 * kTbK) * (th + 2 * kTbK) * 40; }
// Resident blocks per SM the tiled kernels are compiled for (registers: 64
// for 512 threads, 85 for fewer), matching what their shared memory allows
// (64x32: 2, 64x16: 3; the smaller tiles are not limited by it).
constexpr int tb_min_blocks(int nt) { return nt >= 512 ? 2 : nt >= 256 ? 3 : 6; }
constexpr int kGaussTW = 64, kGaussTH = 32, kGaussNT = 256, kGaussMaxR = 15;
constexpr int kIngestNT = 256, kIngestPPT = 8;

// Half-kernel of mask.cpp:225-244 in double on the host.
static GaussTaps make_taps(double sigma) {
    GaussTaps t{};
    const double den = 2 * sigma * sigma;
    const double spi = sigma * std::sqrt(M_PI * 2);
    t.size = (int)(5.0 * sigma) + 1;
    if (t.size > kGaussMaxR + 1) throw Error(OFLOW_ERR_UNSUPPORTED, "Gaussian sigma too large");
    for (int i = 0; i < t.size; i++) t.B[i] = 1 / spi * std::exp(-i * i / den);
    double norm = 0.0;
    for (int i = 0; i < t.size; i++) norm += std::fabs(t.B[i]);
    norm = norm * 2 - t.B[0];
    const double s = 1 / norm;
    for (int i = 0; i < t.size; i++) t.B[i] = s * t.B[i];
    return t;
}

static float zoom_sigma(float zfactor) {
    return (float)(0.6f * std::sqrt(1.0 / (zfactor * zfactor) - 1.0));
}

int tvl1_nscales(int w, int h, int nscales, float zfactor) {
    const float N = (float)(1 + std::log(std::hypot((double)w, (double)h) / 16.0) /
                                    std::log(1 / zfactor));
    return (N < nscales) ? (int)N : nscales;
}

void tvl1_zoom_size(int nx, int ny, int *nxx, int *nyy, float f) {
    *nxx = (int)((float)nx * f + 0.5);
    *nyy = (int)((float)ny * f + 0.5);
}

// ---------------------------------------------------------------- device state
struct TvCtrl {
    int cur;            // state buffer holding the accepted (U, P)
    int n;              // inner iterations done in the current warp
    int stop;           // current warp finished
    unsigned arrive;    // arrival counter of the last-block reduction
    float norm_min, norm_den;
    int norm_apply;
    int redo;           // >0: the next launch re-runs this many iterations (early stop mid-block)
    double energy;
    float last_err;     // error of the last accepted iteration of this warp (inf at its start)
    float decay;        // last_err over the error of the iteration before it
    double pad1[2];
};

// Work queue of the persistent blocked kernel (k_tvl1_q): per pair, the
// claim counter of the current block of K iterations (tiles 0..T-1 are handed
// out in order; claims past T fail), reset by the pair's decision when it
// opens the next block of iterations.  k_warp re-arms it, and the count of
// pairs still running, at the start of every warp stage.
struct TbQueue {
    unsigned long long ticket;
    unsigned long long pad;
};

// Snapshots are written in a launch when the error, extrapolated K-1
// iterations ahead with the last iteration's decay ratio, comes within this
// factor of the threshold: a stop after one of the launch's first K-1
// iterations (the ones a snapshot serves) is plausible.  Elsewhere a stop
// inside a launch falls back to re-running its iterations.  A snapshot launch
// costs about 12 % more than a plain one, a missed stop about one launch of
// the pair; 1.3 measured best among 2.0 (extrapolating K iterations), 2.0
// and 1.3 (K-1 iterations) on the 1024x436 workload.
constexpr float kSnapMargin = 1.3f;

struct NormRec {  // |x|, first index, signed value
    float a;
    int idx;
    float val;
    int pad;
};

__device__ __forceinline__ bool better_max(const NormRec &a, const NormRec &b) {
    return a.a > b.a || (a.a == b.a && a.idx < b.idx);
}
__device__ __forceinline__ bool better_min(const NormRec &a, const NormRec &b) {
    return a.a < b.a || (a.a == b.a && a.idx < b.idx);
}

// The flow state lives in kStateBufs consecutive buffers per quantity (b0 is
// buffer 0, b1 buffer 1, and buffer k starts k*(b1-b0) after b0): 0 and 1
// alternate as the accepted state; 2..4 and 5..7 are two sets of snapshots
// the blocked kernel writes after its first K-1 iterations.  ctrl.cur names
// the buffer that holds the accepted state.
constexpr int kStateBufs = 2 + 2 * (kTbK - 1);
template <typename T> __device__ __forceinline__ T *state_buf(T *b0, T *b1, int k) {
    return b0 + (ptrdiff_t)k * (b1 - b0);
}

// ---------------------------------------------------------------- ingest
// Per-block |x| extrema of both frames of a pair for the normalisation
// (tvl1.cpp:118-123 conversion, :302-317 range), read through the frame table
// (the plan's staging buffers or the caller's pitched device frames); the
// conversion itself happens where the first blur loads the frames.  Indices
// are those of the dense w x h frame, as in the reference.  grid (blocks, B).
template <typename In>
__global__ void __launch_bounds__(kIngestNT) k_ingest(const FrameRef *__restrict__ frames, int w,
                                                      int h, NormRec *recs, int nblk) {
    const int b = blockIdx.y;
    __shared__ NormRec sh[4][kIngestNT / 32];
    NormRec r[4];
    r[0] = {-1.0f, INT_MAX, 0.0f, 0}; r[1] = {INFINITY, INT_MAX, 0.0f, 0};
    r[2] = r[0]; r[3] = r[1];
    // rows blockIdx.x, +nblk, ...: each thread visits its pixels in increasing
    // index order, so a tie keeps the earlier pixel by the strict comparison
    for (int k = 0; k < 2; k++) {
        const FrameRef f = frames[2 * b + k];
        const In *src = static_cast<const In *>(f.p);
        NormRec mx = r[2 * k], mn = r[2 * k + 1];
        for (int y = blockIdx.x; y < h; y += nblk) {
            const In *row = src + (size_t)y * f.pitch;
            for (int xx = threadIdx.x; xx < w; xx += kIngestNT) {
                const float x = (float)__ldg(row + xx);
                const float ax = fabsf(x);
                if (ax > mx.a) mx = NormRec{ax, y * w + xx, x, 0};
                if (ax < mn.a) mn = NormRec{ax, y * w + xx, x, 0};
            }
        }
        r[2 * k] = mx;
        r[2 * k + 1] = mn;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; q++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            NormRec c;
            c.a = __shfl_down_sync(0xffffffffu, r[q].a, o);
            c.idx = __shfl_down_sync(0xffffffffu, r[q].idx, o);
            c.val = __shfl_down_sync(0xffffffffu, r[q].val, o);
            c.pad = 0;
            if ((q & 1) ? better_min(c, r[q]) : better_max(c, r[q])) r[q] = c;
        }
        if (lane == 0) sh[q][wid] = r[q];
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        const int q = threadIdx.x;
        NormRec best = sh[q][0];
        for (int w = 1; w < kIngestNT / 32; w++)
            if ((q & 1) ? better_min(sh[q][w], best) : better_max(sh[q][w], best)) best = sh[q][w];
        recs[((size_t)b * nblk + blockIdx.x) * 4 + q] = best;
    }
}

// One block of 4 warps per pair, warp q reducing quantity q of the per-block
// records: joint range of both frames (std::max / std::min of the per-frame
// |x| extrema, tvl1.cpp:316-321).  (|x|, index) orders the records totally,
// so the result does not depend on the reduction's order.
constexpr int kNormNT = 128;
__global__ void __launch_bounds__(kNormNT) k_norm_finalize(const NormRec *recs, int nblk, TvCtrl *ctrl) {
    const int b = blockIdx.x;
    const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __shared__ NormRec sh[4];
    NormRec best = q & 1 ? NormRec{INFINITY, INT_MAX, 0.0f, 0} : NormRec{-1.0f, INT_MAX, 0.0f, 0};
    for (int i = lane; i < nblk; i += 32) {
        const NormRec c = recs[((size_t)b * nblk + i) * 4 + q];
        if ((q & 1) ? better_min(c, best) : better_max(c, best)) best = c;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        NormRec c;
        c.a = __shfl_down_sync(0xffffffffu, best.a, o);
        c.idx = __shfl_down_sync(0xffffffffu, best.idx, o);
        c.val = __shfl_down_sync(0xffffffffu, best.val, o);
        c.pad = 0;
        if ((q & 1) ? better_min(c, best) : better_max(c, best)) best = c;
    }
    if (lane == 0) sh[q] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        const float a0 = sh[0].val, a1 = sh[2].val, b0 = sh[1].val, b1 = sh[3].val;
        const float mx = (a0 < a1) ? a1 : a0;
        const float mn = (b1 < b0) ? b1 : b0;
        const float den = mx - mn;
        ctrl[b].norm_min = mn;
        ctrl[b].norm_den = den;
        ctrl[b].norm_apply = (den <= 0) ? 0 : 1;  // tvl1.cpp:320-321
        ctrl[b].cur = 0;
        ctrl[b].n = 0;
        ctrl[b].stop = 0;
        ctrl[b].arrive = 0;
        ctrl[b].redo = 0;
    }
}

// ---------------------------------------------------------------- Gaussian
// Separable Gaussian with the reference's mirror (mask.cpp:246-286): rows then
// columns, double taps and sums, each pass rounded to float.  Not in place:
// src planes -> dst planes, gridDim.z = number of planes.  With `normalize`,
// the loaded samples first get 255*(x-min)/den in double (tvl1.cpp:326-327).
__device__ __forceinline__ int gauss_mirror(int x, int n) {
    if (x < 0) return -x;
    if (x >= n) return 2 * n - 1 - x;
    return x;
}

// Fills the LW x LH region sIn (row stride LW) with fetch(ly, lx), NT
// threads as 32 x NT/32: every load of a thread is issued before the first
// store, so they are in flight together.
template <int NT, int LW, int LH, typename F>
__device__ __forceinline__ void load_region(float *sIn, F &&fetch) {
    constexpr int NY = NT / 32, RY = (LH + NY - 1) / NY, RX = (LW + 31) / 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x / 32;
    float v[RY][RX];
#pragma unroll
    for (int a = 0; a < RY; a++)
#pragma unroll
        for (int b = 0; b < RX; b++) {
            const int ly = ty + a * NY, lx = tx + 32 * b;
            v[a][b] = (ly < LH && lx < LW) ? fetch(ly, lx) : 0.0f;
        }
#pragma unroll
    for (int a = 0; a < RY; a++)
#pragma unroll
        for (int b = 0; b < RX; b++) {
            const int ly = ty + a * NY, lx = tx + 32 * b;
            if (ly < LH && lx < LW) sIn[ly * LW + lx] = v[a][b];
        }
}

// Row then column pass of the separable Gaussian over one tile, both with the
// reference's pairing (input[i-j] + input[i+j] in single precision) and double
// taps and sums (mask.cpp:246-286).  RT > 0: the radius at compile time
// (loops unrolled, taps from the parameter bank); RT = 0: taps.size - 1.
template <int RT>
__device__ __forceinline__ double gauss_sum(const float *c, int step, const GaussTaps &taps, int R) {
    double sum = taps.B[0] * (double)c[0];
    if (RT > 0) {
#pragma unroll
        for (int j = 1; j <= RT; j++) {
            const float pair = c[-j * step] + c[j * step];
            sum += taps.B[j] * (double)pair;
        }
    } else {
        for (int j = 1; j <= R; j++) {
            const float pair = c[-j * step] + c[j * step];
            sum += taps.B[j] * (double)pair;
        }
    }
    return sum;
}

// SRC 0: float planes at src; 1 / 2: uint8 / float frames through the frame
// table (plane z = frame z of the table), converted to float on load.  A
// uint8 frame is normalised through a 256-entry table of the same expression.
// Tile kGaussTW x kGaussTH outputs, 256 threads as 32 x 8.
template <int SRC, int RT>
__global__ void __launch_bounds__(kGaussNT) k_gauss(const float *__restrict__ src, float *dst,
                                                    int nx, int ny, size_t plane_stride,
                                                    GaussTaps taps, const TvCtrl *ctrl,
                                                    int normalize, const FrameRef *frames) {
    constexpr int MR = RT > 0 ? RT : kGaussMaxR;
    constexpr int LW = kGaussTW + 2 * MR, LH = kGaussTH + 2 * MR;
    __shared__ float sIn[LH * LW];
    __shared__ float sRow[LH * kGaussTW];
    __shared__ float sLut[SRC == 1 ? 256 : 1];
    const int R = RT > 0 ? RT : taps.size - 1;
    const int z = blockIdx.z;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const float *in = src + (size_t)z * plane_stride;
    float *out = dst + (size_t)z * plane_stride;
    const int x0 = blockIdx.x * kGaussTW, y0 = blockIdx.y * kGaussTH;
    bool apply = false;
    float mn = 0.0f, den = 1.0f;
    if (normalize) {
        const TvCtrl &c = ctrl[z >> 1];
        apply = c.norm_apply != 0;
        mn = c.norm_min;
        den = c.norm_den;
    }
    FrameRef f{};
    if (SRC != 0) f = frames[z];
    if (SRC == 1) {
        const float v = (float)threadIdx.x;
        sLut[threadIdx.x] = apply ? (float)(255.0 * (double)(v - mn) / (double)den) : v;
        __syncthreads();
    }
    const int lw = kGaussTW + 2 * R, lh = kGaussTH + 2 * R;
    auto fetch = [&](int ly, int lx) -> float {
        const int my = gauss_mirror(y0 - R + ly, ny), mx = gauss_mirror(x0 - R + lx, nx);
        if (my < 0 || my >= ny || mx < 0 || mx >= nx) return 0.0f;
        if (SRC == 0) return __ldg(in + (size_t)my * nx + mx);
        if (SRC == 1) return sLut[__ldg(static_cast<const uint8_t *>(f.p) + (size_t)my * f.pitch + mx)];
        float v = __ldg(static_cast<const float *>(f.p) + (size_t)my * f.pitch + mx);
        if (apply) v = (float)(255.0 * (double)(v - mn) / (double)den);
        return v;
    };
    if (RT > 0)
        load_region<kGaussNT, LW, LH>(sIn, fetch);
    else
        for (int ly = ty; ly < lh; ly += kGaussNT / 32)
            for (int lx = tx; lx < lw; lx += 32) sIn[ly * LW + lx] = fetch(ly, lx);
    __syncthreads();
    for (int ly = ty; ly < lh; ly += kGaussNT / 32)
        for (int cx = tx; cx < kGaussTW; cx += 32)
            sRow[ly * kGaussTW + cx] = (float)gauss_sum<RT>(sIn + ly * LW + cx + R, 1, taps, R);
    __syncthreads();
    for (int cy = ty; cy < kGaussTH; cy += kGaussNT / 32) {
        const int y = y0 + cy;
        if (y >= ny) break;
        for (int cx = tx; cx < kGaussTW; cx += 32) {
            const int x = x0 + cx;
            if (x >= nx) break;
            out[(size_t)y * nx + x] =
                (float)gauss_sum<RT>(sRow + (cy + R) * kGaussTW + cx, kGaussTW, taps, R);
        }
    }
}

// zoom_out at factor 1/2 (zoom.cpp:20-53) in one pass: the blur of k_gauss<0>
// evaluated only where the bicubic resample reads it.  At factor 1/2 the
// sample of output (j, i) is taken at (2j, 2i) exactly, where the Keys cubic
// returns its centre tap unchanged (offset 0), so the level is the blurred
// plane at the even rows and columns: the row pass runs on even columns only
// and the column pass on even rows only, with the same taps, mirror, pairing
// and double sums as k_gauss, so every output is bit-identical to blur then
// resample.  Tile: kDecTW x kDecTH outputs, 256 threads as 32 x 8; gridDim.z
// = planes.
constexpr int kDecTW = 32, kDecTH = 32, kDecNT = 256, kDecMaxR = 8;
template <int RT>
__global__ void __launch_bounds__(kDecNT) k_gauss_dec2(const float *__restrict__ src, size_t src_stride,
                                                       int nx, int ny, float *dst, size_t dst_stride,
                                                       int nxx, int nyy, GaussTaps taps) {
    constexpr int MR = RT > 0 ? RT : kDecMaxR;
    constexpr int LW = 2 * kDecTW - 1 + 2 * MR, LH = 2 * kDecTH - 1 + 2 * MR;
    __shared__ float sIn[LH * LW];
    __shared__ float sRow[LH * kDecTW];
    const int R = RT > 0 ? RT : taps.size - 1;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const float *in = src + (size_t)blockIdx.z * src_stride;
    float *out = dst + (size_t)blockIdx.z * dst_stride;
    const int x0 = blockIdx.x * kDecTW, y0 = blockIdx.y * kDecTH;
    const int ix0 = 2 * x0 - R, iy0 = 2 * y0 - R;  // input origin of the region
    const int lw = 2 * kDecTW - 1 + 2 * R, lh = 2 * kDecTH - 1 + 2 * R;
    auto fetch = [&](int ly, int lx) -> float {
        const int my = gauss_mirror(iy0 + ly, ny), mx = gauss_mirror(ix0 + lx, nx);
        if (my < 0 || my >= ny || mx < 0 || mx >= nx) return 0.0f;
        return __ldg(in + (size_t)my * nx + mx);
    };
    if (RT > 0)
        load_region<kDecNT, LW, LH>(sIn, fetch);
    else
        for (int ly = ty; ly < lh; ly += kDecNT / 32)
            for (int lx = tx; lx < lw; lx += 32) sIn[ly * LW + lx] = fetch(ly, lx);
    __syncthreads();
    for (int ly = ty; ly < lh; ly += kDecNT / 32)
        sRow[ly * kDecTW + tx] = (float)gauss_sum<RT>(sIn + ly * LW + 2 * tx + R, 1, taps, R);
    __syncthreads();
    const int x = x0 + tx;
    if (x >= nxx) return;
    for (int cy = ty; cy < kDecTH; cy += kDecNT / 32) {
        const int y = y0 + cy;
        if (y >= nyy) break;
        out[(size_t)y * nxx + x] =
            (float)gauss_sum<RT>(sRow + (2 * cy + R) * kDecTW + tx, kDecTW, taps, R);
    }
}

// ---------------------------------------------------------------- resampling
// Bicubic resample without border zeroing (zoom.cpp:20-53 and :61-85):
// out(j, i) = in((float)j / dx, (float)i / dy).  gridDim.z = planes.
__global__ void k_resample(const float *__restrict__ src, size_t src_stride, int nx, int ny,
                           float *dst, size_t dst_stride, int nxx, int nyy, float dx, float dy) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= nxx || i >= nyy) return;
    const float *in = src + (size_t)blockIdx.z * src_stride;
    const float i2 = (float)i / dy, j2 = (float)j / dx;
    dst[(size_t)blockIdx.z * dst_stride + (size_t)i * nxx + j] = bicubic_at(in, j2, i2, nx, ny, false);
}

// Flow upsampling to the next finer scale (tvl1.cpp:167-172): bicubic of both
// components at (j*nx/nxx, i*ny/nyy) then times 1/zfactor.  Reads U[cur].
// Each thread writes the outputs j0 = 2*tid and j0 + 1 of one row: they share
// ty, and at a zoom factor of 2 also the stencil, so the four columns' first
// passes are evaluated once for both (a pair whose stencils differ takes them
// separately).
__device__ __forceinline__ void zoom_columns(const float2 *U, int nx, const BicubicStencil &s,
                                             float *a, float *c) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float2 *col = U + s.col[k];
        const float2 t0 = col[(size_t)nx * s.row[0]], t1 = col[(size_t)nx * s.row[1]];
        const float2 t2 = col[(size_t)nx * s.row[2]], t3 = col[(size_t)nx * s.row[3]];
        a[k] = cubic_cell(t0.x, t1.x, t2.x, t3.x, s.ty);
        c[k] = cubic_cell(t0.y, t1.y, t2.y, t3.y, s.ty);
    }
}

__global__ void k_zoom_flow(const float2 *U0, const float2 *U1, size_t stride, int nx, int ny,
                            float2 *Uz, int nxx, int nyy, float fx, float fy, float inv,
                            const TvCtrl *ctrl) {
    const int j0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    const int b = blockIdx.z;
    if (j0 >= nxx || i >= nyy) return;
    const float2 *U = state_buf(U0, U1, ctrl[b].cur) + (size_t)b * stride;
    float2 *out = Uz + (size_t)b * stride + (size_t)i * nxx;
    const float i2 = (float)i / fy;
    BicubicStencil s0;
    bicubic_stencil((float)j0 / fx, i2, nx, ny, false, s0);
    float a[4], c[4];
    zoom_columns(U, nx, s0, a, c);
    out[j0] = make_float2(inv * cubic_cell(a[0], a[1], a[2], a[3], s0.tx),
                          inv * cubic_cell(c[0], c[1], c[2], c[3], s0.tx));
    const int j1 = j0 + 1;
    if (j1 >= nxx) return;
    BicubicStencil s1;
    bicubic_stencil((float)j1 / fx, i2, nx, ny, false, s1);
    if (s1.col[0] != s0.col[0] || s1.col[1] != s0.col[1] || s1.col[2] != s0.col[2] ||
        s1.col[3] != s0.col[3])
        zoom_columns(U, nx, s1, a, c);
    out[j1] = make_float2(inv * cubic_cell(a[0], a[1], a[2], a[3], s1.tx),
                          inv * cubic_cell(c[0], c[1], c[2], c[3], s1.tx));
}

// ---------------------------------------------------------------- gradient
// Centered gradient of I1 (mask.cpp:139-196) at (x, y), packed with I1
// itself: (I1, I1x, I1y).
__device__ __forceinline__ float3 grad_at(const float *__restrict__ I, int x, int y, int nx, int ny) {
    const size_t row = (size_t)y * nx;
    const float ddx = __ldg(I + row + imin(x + 1, nx - 1)) - __ldg(I + row + imax(x - 1, 0));
    const float ddy = __ldg(I + (size_t)imin(y + 1, ny - 1) * nx + x) -
                      __ldg(I + (size_t)imax(y - 1, 0) * nx + x);
    return make_float3(__ldg(I + row + x), (float)(0.5 * (double)ddx), (float)(0.5 * (double)ddy));
}

// Column coefficients of the warp's bicubic samples, once per scale.  A
// sample that is not zeroed at the border has rows y-1..y+2 and columns
// x-1..x+2 of its base texel (x, y) (bicubic_stencil: a negative coordinate
// always reaches outside, so both steps are +1), and its first pass evaluates
// the column cubic of rows y-1..y+2 at ty for each of the four columns.  The
// part of that cubic that does not depend on ty (cubic_coef) is computed here
// for every texel (x, y) and each of I1, I1x, I1y; the warp then evaluates it
// (cubic_eval) with the same operations in the same order.  Rows outside
// [1, ny-3] are never read by a sample; they hold the coefficients of the
// clamped rows.
__global__ void k_cubic_pack(const float *__restrict__ pyr, size_t pyr_stride, int nx, int ny,
                             WarpCoef wc, size_t stride) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int b = blockIdx.z;
    if (x >= nx || y >= ny) return;
    const float *I = pyr + (size_t)(2 * b + 1) * pyr_stride;
    float3 g[4];
#pragma unroll
    for (int r = 0; r < 4; r++) g[r] = grad_at(I, x, imin(imax(y - 1 + r, 0), ny - 1), nx, ny);
    const CubicCoef k0 = cubic_coef(g[0].x, g[1].x, g[2].x, g[3].x);
    const CubicCoef k1 = cubic_coef(g[0].y, g[1].y, g[2].y, g[3].y);
    const CubicCoef k2 = cubic_coef(g[0].z, g[1].z, g[2].z, g[3].z);
    const size_t q = (size_t)b * stride + (size_t)y * nx + x;
    wc.cc0[q] = make_double2(k0.c3, k0.c2);
    wc.cc1[q] = make_double2(k1.c3, k1.c2);
    wc.cc2[q] = make_double2(k2.c3, k2.c2);
    wc.dv01[q] = make_float4(k0.d20, k0.v1, k1.d20, k1.v1);
    wc.dv2[q] = make_float2(k2.d20, k2.v1);
}

// ---------------------------------------------------------------- warping
// Per warp (tvl1.cpp:197-212): bicubic samples of I1, I1x, I1y at (x+u1,
// y+u2) with border zeroing, then rho_c and |grad I1w|^2 (tvl1.cpp:202-212),
// packed as one float4 per pixel.  mode 0: u from U[cur];
// 1: u from the upsampled Uz (copied into U[cur]); 2: u = 0 (coarsest scale).
// With first_warp, p is zeroed (tvl1.cpp:190-193).
enum { kWarpFromU = 0, kWarpFromUz = 1, kWarpZero = 2 };

// The first pass of each sample reads the column coefficients of its four
// columns (k_cubic_pack) and evaluates them at ty; only the second pass runs
// the whole cell.  6 blocks of 256 per SM: the gathers need the warps to hide
// their latency.  Splitting the channels over three threads per pixel (all
// eight gathers of a channel in flight, the samples combined in shared
// memory) measured slower: 4.10 against 2.48 ms for the 25 warps of the
// 1024x436 workload at 32 pairs.
constexpr int kWarpTW = 32, kWarpTH = 8;
__global__ void __launch_bounds__(kWarpTW * kWarpTH, 6) k_warp(const float *__restrict__ pyr, size_t pyr_stride, WarpCoef wc,
                       float4 *WR, float2 *U0, float2 *U1, const float2 *Uz, float4 *P0,
                       float4 *P1, size_t stride, int nx, int ny, int mode, int first_warp,
                       TvCtrl *ctrl, TbQueue *q, int *left) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int b = blockIdx.z;
    if (x == 0 && y == 0) {
        ctrl[b].n = 0;
        ctrl[b].stop = 0;
        ctrl[b].arrive = 0;
        ctrl[b].redo = 0;
        ctrl[b].last_err = INFINITY;
        ctrl[b].decay = 1.0f;
        q[b].ticket = 0;  // the persistent form's work queue, re-armed per stage
        if (b == 0) *left = gridDim.z;
    }
    if (x >= nx || y >= ny) return;
    const int cur = ctrl[b].cur;
    const size_t off = (size_t)b * stride, p = (size_t)y * nx + x;
    float2 *U = state_buf(U0, U1, cur) + off;
    float2 u;
    if (mode == kWarpFromU) {
        u = U[p];
    } else if (mode == kWarpFromUz) {
        u = Uz[off + p];
        U[p] = u;
    } else {
        u = make_float2(0.0f, 0.0f);
        U[p] = u;
    }
    if (first_warp) (state_buf(P0, P1, cur) + off)[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float uu = (float)x + u.x, vv = (float)y + u.y;
    float Iw = 0.0f, Iwx = 0.0f, Iwy = 0.0f;
    BicubicStencil s;
    if (bicubic_stencil(uu, vv, nx, ny, true, s)) {
        // base texel (col[1], row[1]); columns col[1]-1 .. col[1]+2
        const size_t q0 = off + (size_t)nx * s.row[1] + s.col[0];
        const double ty = s.ty, hy = 0.5 * ty;
        float a[4], bx[4], by[4];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const size_t q = q0 + c;
            const double2 k0 = __ldg(wc.cc0 + q), k1 = __ldg(wc.cc1 + q), k2 = __ldg(wc.cc2 + q);
            const float4 d01 = __ldg(wc.dv01 + q);
            const float2 d2 = __ldg(wc.dv2 + q);
            a[c] = cubic_eval(k0.x, k0.y, d01.x, d01.y, ty, hy);
            bx[c] = cubic_eval(k1.x, k1.y, d01.z, d01.w, ty, hy);
            by[c] = cubic_eval(k2.x, k2.y, d2.x, d2.y, ty, hy);
        }
        Iw = cubic_cell(a[0], a[1], a[2], a[3], s.tx);
        Iwx = cubic_cell(bx[0], bx[1], bx[2], bx[3], s.tx);
        Iwy = cubic_cell(by[0], by[1], by[2], by[3], s.tx);
    }
    const float I0v = __ldg(pyr + (size_t)(2 * b) * pyr_stride + p);
    const float rho_c = (Iw - Iwx * u.x - Iwy * u.y - I0v);
    WR[off + p] = make_float4(Iwx, Iwy, rho_c, (Iwx * Iwx) + (Iwy * Iwy));
}

// ---------------------------------------------------------------- iteration
// Divergence of (a1, a2) at one pixel from its value c and its left / upper
// neighbours, with the border forms and evaluation order of mask.cpp:31-90.
__device__ __forceinline__ float div_border(float a1c, float a1l, float a2c, float a2u, bool L,
                                            bool R, bool T, bool B) {
    if (!(L | R | T | B)) return (a1c - a1l) + (a2c - a2u);
    if (T && !L && !R) return a1c - a1l + a2c;
    if (B && !L && !R) return a1c - a1l - a2u;
    if (L && !T && !B) return a1c + a2c - a2u;
    if (R && !T && !B) return -a1l + a2c - a2u;
    if (L && T) return a1c + a2c;
    if (R && T) return -a1l + a2c;
    if (L && B) return a1c - a2u;
    return -a1l - a2u;
}

// TH step (tvl1.cpp:221-245) and u update (:252-265) for one pixel.  wr holds
// (I1wx, I1wy, rho_c, |grad I1w|^2).  The branches of the reference pick the
// coefficient of (I1wx, I1wy): l_t where rho < -l_t*grad, -l_t where rho >
// l_t*grad, 0 where the gradient vanishes, else -rho/grad; the products are
// the reference's, so the result is identical.  The quotient is formed for
// every pixel (most need it) by Markstein's correction from RN(1/grad), which
// equals IEEE division inside the ranges rcp_in_range and markstein_safe
// cover; a pixel that needs the quotient outside them takes the division.
__device__ __forceinline__ float2 th_u_update(float2 u, float4 wr, float4 pc, float4 pl, float4 pu,
                                              bool L, bool R, bool T, bool B, float l_t,
                                              float theta) {
    const float grad = wr.w;
    const float rho = wr.z + (wr.x * u.x + wr.y * u.y);
    const float lg = l_t * grad;
    const bool c1 = rho >= -lg, c2 = rho > lg, c3 = grad < 1E-10f;
    const float nrho = -rho;
    float fi = markstein(nrho, grad, rcp_near_rn(grad));
    if (c1 && !c2 && !c3 && !(rcp_in_range(grad) && markstein_safe(nrho))) fi = nrho / grad;
    const float k = !c1 ? l_t : (c2 ? -l_t : fi);
    const bool flat = c1 && !c2 && c3;  // the reference's d = 0, by selection
    const float d1 = flat ? 0.0f : k * wr.x, d2 = flat ? 0.0f : k * wr.y;
    const float v1 = u.x + d1, v2 = u.y + d2;
    const float div1 = div_border(pc.x, pl.x, pc.y, pu.y, L, R, T, B);
    const float div2 = div_border(pc.z, pl.z, pc.w, pu.w, L, R, T, B);
    return make_float2(v1 + theta * div1, v2 + theta * div2);
}

// Dual update (tvl1.cpp:268-291) from the forward differences of u(new):
// g = 1 + tau/theta*hypot(grad u), p = (p + tau/theta*grad u) / g, with the
// hypot as glibc computes it (hypot_ref) and the divisions by Markstein's
// correction from RN(1/g) (exact_math.cuh).  The conditions of the Markstein
// form are checked without branching; a pixel outside them takes the IEEE
// divisions in one shared branch.
__device__ __forceinline__ float4 dual_update(float4 po, float f1x, float f1y, float f2x,
                                              float f2y, float taut) {
    const float g1 = 1.0f + taut * hypot_ref(f1x, f1y);
    const float g2 = 1.0f + taut * hypot_ref(f2x, f2y);
    const float r1 = rcp_near_rn(g1), r2 = rcp_near_rn(g2);
    const float n1 = taut * f1x + po.x, n2 = taut * f1y + po.y;
    const float n3 = taut * f2x + po.z, n4 = taut * f2y + po.w;
    float4 pn;
    pn.x = markstein(n1, g1, r1);
    pn.y = markstein(n2, g1, r1);
    pn.z = markstein(n3, g2, r2);
    pn.w = markstein(n4, g2, r2);
    const bool fast = rcp_in_range(g1) && rcp_in_range(g2) && markstein_safe(n1) &&
                      markstein_safe(n2) && markstein_safe(n3) && markstein_safe(n4);
    if (!fast) {
        pn.x = n1 / g1;
        pn.y = n2 / g1;
        pn.z = n3 / g2;
        pn.w = n4 / g2;
    }
    return pn;
}

struct IterArgs {
    const float4 *WR;  // (I1wx, I1wy, rho_c, |grad I1w|^2) per pixel
    float2 *U0, *U1;
    float4 *P0, *P1;
    size_t stride;  // elements between pairs
    int nx, ny;
    float l_t, theta, taut, eps2;
    TvCtrl *ctrl;
    double *partials;  // [B][max_blocks]
    int max_blocks;
    int *iters;        // [B][iter_stride]
    int iter_stride, stage;
};

// One inner iteration (tvl1.cpp:218-291) on a TW x TH tile:
//  A: p(old) on the tile plus a one-pixel ring -> smem
//  B: TH step, divergence and u update on the tile plus one column to the
//     right and one row below (those are recomputed by the neighbour tile the
//     same way), u(new) -> smem; owned pixels add their squared change
//  C: forward gradient of u(new), g = 1 + tau/theta*|grad u|, p update.
// The last block of a pair finishes the error reduction and the loop control.
template <int TW, int TH, int NT>
__global__ void __launch_bounds__(NT) k_tvl1_iter(IterArgs a) {
    const int b = blockIdx.z;
    TvCtrl *ctrl = a.ctrl + b;
    if (*((volatile int *)&ctrl->stop)) return;
    const int cur = *((volatile int *)&ctrl->cur);
    const int nx = a.nx, ny = a.ny;
    const size_t off = (size_t)b * a.stride;
    const float2 *__restrict__ Uin = state_buf(a.U0, a.U1, cur) + off;
    float2 *__restrict__ Uout = state_buf(a.U0, a.U1, cur ^ 1) + off;
    const float4 *__restrict__ Pin = state_buf(a.P0, a.P1, cur) + off;
    float4 *__restrict__ Pout = state_buf(a.P0, a.P1, cur ^ 1) + off;
    const float4 *__restrict__ WR = a.WR + off;
    const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;

    __shared__ float4 sP[(TH + 2) * (TW + 2)];
    __shared__ float2 sU[(TH + 1) * (TW + 1)];
    __shared__ double sred[NT / 32];
    __shared__ int s_last;

    for (int i = threadIdx.x; i < (TH + 2) * (TW + 2); i += NT) {
        const int x = x0 + i % (TW + 2) - 1, y = y0 + i / (TW + 2) - 1;
        float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
        if (x >= 0 && x < nx && y >= 0 && y < ny) p = Pin[(size_t)y * nx + x];
        sP[i] = p;
    }
    __syncthreads();

    double err = 0.0;
    for (int i = threadIdx.x; i < (TH + 1) * (TW + 1); i += NT) {
        const int rx = i % (TW + 1), ry = i / (TW + 1);
        const int x = x0 + rx, y = y0 + ry;
        if (x >= nx || y >= ny) continue;
        const size_t p = (size_t)y * nx + x;
        const float2 u = Uin[p];
        const float4 *c = sP + (ry + 1) * (TW + 2) + (rx + 1);
        const float2 un = th_u_update(u, WR[p], c[0], c[-1], c[-(TW + 2)], x == 0,
                                      x == nx - 1, y == 0, y == ny - 1, a.l_t, a.theta);
        sU[i] = un;
        if (rx < TW && ry < TH) {
            Uout[p] = un;
            const float e1 = un.x - u.x, e2 = un.y - u.y;
            const float term = e1 * e1 + e2 * e2;
            err += (double)term;
        }
    }
    __syncthreads();

    for (int i = threadIdx.x; i < TW * TH; i += NT) {
        const int rx = i % TW, ry = i / TW;
        const int x = x0 + rx, y = y0 + ry;
        if (x >= nx || y >= ny) continue;
        const float2 uc = sU[ry * (TW + 1) + rx];
        float f1x = 0.0f, f2x = 0.0f, f1y = 0.0f, f2y = 0.0f;
        if (x < nx - 1) {
            const float2 ur = sU[ry * (TW + 1) + rx + 1];
            f1x = ur.x - uc.x;
            f2x = ur.y - uc.y;
        }
        if (y < ny - 1) {
            const float2 ud = sU[(ry + 1) * (TW + 1) + rx];
            f1y = ud.x - uc.x;
            f2y = ud.y - uc.y;
        }
        const float4 pn = dual_update(sP[(ry + 1) * (TW + 2) + rx + 1], f1x, f1y, f2x, f2y, a.taut);
        Pout[(size_t)y * nx + x] = pn;
    }

    // ---- error reduction and loop control (tvl1.cpp:252-265, :216)
    const double bsum = block_sum_double<NT>(err, sred);
    const int nblk = gridDim.x * gridDim.y;
    double *part = a.partials + (size_t)b * a.max_blocks;
    if (threadIdx.x == 0) {
        part[blockIdx.y * gridDim.x + blockIdx.x] = bsum;
        __threadfence();
        const unsigned prev = atomicAdd(&ctrl->arrive, 1u);
        s_last = (prev == (unsigned)nblk - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double acc = 0.0;
    for (int k = threadIdx.x; k < nblk; k += NT) acc += __ldcg(part + k);
    const double tot = block_sum_double<NT>(acc, sred);
    if (threadIdx.x == 0) {
        float e = (float)tot;
        e = e / (float)(nx * ny);
        const int n = ctrl->n + 1;
        ctrl->n = n;
        a.iters[(size_t)b * a.iter_stride + a.stage] = n;
        ctrl->cur = cur ^ 1;
        if (!(e > a.eps2)) ctrl->stop = 1;
        ctrl->arrive = 0;
        __threadfence();
    }
}


// ---------------------------------------------------------------- blocked iterations
// Up to K inner iterations per launch on a TW x TH tile held in shared memory
// with a K-pixel halo (the dependency cone of one iteration is one pixel in
// every direction, so after K iterations the owned tile is exact).  The state
// is loaded once and stored once per launch, so HBM traffic per iteration
// drops by about K.  Each iteration's squared change over the owned pixels is
// kept; the last block of a pair finds the first iteration that meets the
// stopping rule (tvl1.cpp:216).  When a stop is plausible (kSnapMargin), the
// owned tile is also stored after each of the first K-1 iterations into a
// snapshot buffer, so a stop in the middle of the launch accepts that
// iteration's state; otherwise the next launch re-runs those iterations.
struct TbArgs {
    const float4 *WR;
    float2 *U0, *U1;
    float4 *P0, *P1;
    size_t stride;
    int nx, ny, max_it;
    float l_t, theta, taut, eps2;
    TvCtrl *ctrl;
    double *partials;  // [B][max_tiles][K]
    int max_tiles;
    int *iters;
    int iter_stride, stage;
    // TMA region loads (k_tvl1_tb): use_tma set when the maps below describe
    // this level for the launched tile shape; err is set when a load's
    // bounded wait gives up
    int use_tma;
    int *err;
    // queue form only: size a pair's block of iterations to end where the
    // error's geometric decay predicts its stop (the launch form's fixed
    // schedule needs full blocks)
    int predict;
    CUtensorMap tmP;  // p: (2 nx, ny, pair, buffer) 8-byte elements
    CUtensorMap tmU;  // u: (nx, ny, pair, buffer) 8-byte elements
    CUtensorMap tmW;  // (I1wx, I1wy, rho_c, grad): (2 nx, ny, pair) 8-byte elements
};

// One blocked iteration j (1-based) over the region.  Phase B (TH + u update)
// covers [j, RW-j]^2 and phase C (dual update) [j, RW-1-j]^2: exactly the
// pixels whose values reach the owned tile after K iterations, so no read
// ever leaves the region.  INTERIOR: no region pixel lies on the image border
// (no bounds or border tests).
template <int TW, int TH, int K, int NT, bool INTERIOR>
__device__ __forceinline__ void tb_iteration(int j, float4 *sP, const float4 *sWR, float2 *sU, int ox, int oy, int nx,
                                             int ny, float l_t, float theta, float taut,
                                             double &err) {
    constexpr int RW = TW + 2 * K, RH = TH + 2 * K;
    for_rect<NT>(j, RW - j, j, RH - j, [&](int rx, int ry) {
        const int i = ry * RW + rx;
        const int x = ox + rx, y = oy + ry;
        if (!INTERIOR && (x >= nx || y >= ny || x < 0 || y < 0)) return;
        const float2 u = sU[i];
        const float2 un = th_u_update(u, sWR[i], sP[i], sP[i - 1], sP[i - RW],
                                      !INTERIOR && x == 0, !INTERIOR && x == nx - 1,
                                      !INTERIOR && y == 0, !INTERIOR && y == ny - 1, l_t, theta);
        sU[i] = un;
        if (rx >= K && rx < K + TW && ry >= K && ry < K + TH) {
            const float e1 = un.x - u.x, e2 = un.y - u.y;
            const float term = e1 * e1 + e2 * e2;
            err += (double)term;
        }
    });
    __syncthreads();
    for_rect<NT>(j, RW - 1 - j, j, RH - 1 - j, [&](int rx, int ry) {
        const int i = ry * RW + rx;
        const int x = ox + rx, y = oy + ry;
        if (!INTERIOR && (x >= nx || y >= ny || x < 0 || y < 0)) return;
        const float2 uc = sU[i];
        float f1x = 0.0f, f2x = 0.0f, f1y = 0.0f, f2y = 0.0f;
        if (INTERIOR || x < nx - 1) {
            const float2 ur = sU[i + 1];
            f1x = ur.x - uc.x;
            f2x = ur.y - uc.y;
        }
        if (INTERIOR || y < ny - 1) {
            const float2 ud = sU[i + RW];
            f1y = ud.x - uc.x;
            f2y = ud.y - uc.y;
        }
        sP[i] = dual_update(sP[i], f1x, f1y, f2x, f2y, taut);
    });
    __syncthreads();
}

// Per-iteration error sums of one block into its partial slots, then the
// stopping decision by the last block of the pair to arrive: it finds the
// first of the kk iterations meeting the stopping rule (tvl1.cpp:216) and
// accepts the state after that iteration -- the final buffer, or the snapshot
// written after it (snap >= 0).  Without a snapshot, `redo` makes the next
// launch re-run exactly that many iterations from the untouched input.  The
// result is that of one iteration per launch either way.  Partials are summed
// in a fixed order, so the decision does not depend on block scheduling.
// Dynamic shared memory the decision may reuse once the tile is stored: K x
// (NT/32) doubles.  (Static shared memory is kept small: two 64x32 tiles per
// SM leave it under 512 bytes a block.)
template <int K, int NT>
__device__ __forceinline__ bool tb_decide(const TbArgs &a, TvCtrl *ctrl, int b, int tile,
                                          int ntiles, double wsum, int kk, int fin,
                                          int snap, int redo, int n0, TbQueue *q, int *left,
                                          double *scratch) {
    // The K sums share one block barrier: per warp a fixed shuffle tree, then
    // thread 0 adds the warps in order (block_sum_double's order, per sum).
    constexpr int NW = NT / 32;
    double(*sred)[NW] = reinterpret_cast<double(*)[NW]>(scratch);
    __shared__ double sE[K];
    __shared__ int s_last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double *part = a.partials + (size_t)b * a.max_tiles * K;
    __syncthreads();  // every thread has stored its share of the tile (scratch overlays it)
    if (lane < K) sred[lane][wid] = wsum;  // the warp sums of tb_tile (lane j: iteration j)
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int j = 0; j < kk; j++) {
            double r = 0.0;
#pragma unroll
            for (int w = 0; w < NW; w++) r += sred[j][w];
            part[(size_t)tile * K + j] = r;
        }
        __threadfence();
        const unsigned prev = atomicAdd(&ctrl->arrive, 1u);
        s_last = (prev == (unsigned)ntiles - 1);
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    {
        double acc[K];
#pragma unroll
        for (int j = 0; j < K; j++) acc[j] = 0.0;
        for (int t = threadIdx.x; t < ntiles; t += NT)
#pragma unroll
            for (int j = 0; j < K; j++)
                if (j < kk) acc[j] += __ldcg(part + (size_t)t * K + j);
#pragma unroll
        for (int j = 0; j < K; j++) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[j] += __shfl_down_sync(0xffffffffu, acc[j], o);
            if (lane == 0) sred[j][wid] = acc[j];
        }
        __syncthreads();
        if (threadIdx.x == 0)
            for (int j = 0; j < kk; j++) {
                double r = 0.0;
#pragma unroll
                for (int w = 0; w < NW; w++) r += sred[j][w];
                sE[j] = r;
            }
    }
    if (threadIdx.x == 0) {
        const float npx = (float)(a.nx * a.ny);
        if (redo > 0) {  // the re-run ends exactly at the stopping iteration
            ctrl->n = n0 + redo;
            ctrl->cur = fin;
            ctrl->stop = 1;
            ctrl->redo = 0;
        } else if (kk <= 0) {  // no iterations left (max_it reached or 0)
            ctrl->stop = 1;
        } else {
            int stopj = 0;
            float e_last = INFINITY, e_prev = INFINITY;
            for (int j = 0; j < kk; j++) {
                float e = (float)sE[j];
                e = e / npx;
                e_prev = e_last;
                e_last = e;
                if (!(e > a.eps2) || n0 + j + 1 >= a.max_it) {
                    stopj = j + 1;
                    break;
                }
            }
            if (stopj == 0 || stopj == kk) {
                ctrl->n = n0 + kk;
                ctrl->cur = fin;
                ctrl->last_err = e_last;
                ctrl->decay = (e_prev > 0.0f && e_prev < INFINITY) ? e_last / e_prev : 1.0f;
                if (stopj) ctrl->stop = 1;
            } else if (snap >= 0) {
                // a stop after iteration stopj < kk accepts that iteration's snapshot
                ctrl->n = n0 + stopj;
                ctrl->cur = snap + stopj - 1;
                ctrl->stop = 1;
            } else {
                ctrl->redo = stopj;  // no snapshot: re-run stopj iterations next launch
            }
        }
        a.iters[(size_t)b * a.iter_stride + a.stage] = ctrl->n;
        ctrl->arrive = 0;
        __threadfence();
        if (q) {
            // the decision is visible before the next block of iterations opens
            if (ctrl->stop) atomicSub(left, 1);
            else atomicExch(&q[b].ticket, 0ull);
        }
    }
    return true;
}

// Reads the control block of pair b at the start of a block of iterations:
// the accepted buffer, iterations done, re-run count, and whether snapshots
// are due (kSnapMargin).  `fresh`: read past L1 (the persistent kernel sees
// the block change between its tiles).
struct TbStart {
    int cur, n0, redo, kk;
    bool snaps;
};
template <int K>
__device__ __forceinline__ TbStart tb_start(const TbArgs &a, const TvCtrl *ctrl) {
    TbStart t;
    t.cur = __ldcg(&ctrl->cur);
    t.n0 = __ldcg(&ctrl->n);
    t.redo = __ldcg(&ctrl->redo);
    t.kk = t.redo > 0 ? t.redo : imin(K, a.max_it - t.n0);
    t.snaps = false;
    if (t.redo == 0) {
        const float q = fminf(__ldcg(&ctrl->decay), 1.0f);
        const float le = __ldcg(&ctrl->last_err);
        float qk = 1.0f;
#pragma unroll
        for (int j = 1; j < K; j++) qk *= q;
        t.snaps = le * qk < kSnapMargin * a.eps2;
        if (a.predict && q > 0.0f && q < 1.0f && le > a.eps2 && le < INFINITY) {
            // iterations until le * q^n <= eps2; the same inputs give every
            // tile of the pair the same count
            const float n = ceilf(logf(a.eps2 / le) / logf(q));
            if (n >= 1.0f && n < (float)t.kk) {
                t.kk = (int)n;
                // predict 2: trust the prediction, no snapshots (an earlier
                // stop re-runs its iterations); measured 1,234 against 1,225
                // pairs/s with snapshots, 1,176 with full blocks
                if (a.predict == 2) t.snaps = false;
            }
        }
    }
    return t;
}

// One tile of one pair for kk <= K iterations: the region in (TMA boxes on
// `bar` with the given phase parity, or plain loads past L1), the iterations,
// the snapshot stores and the final store of the owned tile.  The owned
// pixels' squared change of iteration j is summed over each warp right after
// the iteration (the fixed shuffle tree tb_decide applies) and lane j keeps
// the warp's sum in wsum, so no per-iteration accumulator stays live across
// the iterations.  Returns false if the TMA wait gave up (the error flag is
// set; the caller leaves).
template <int TW, int TH, int K, int NT>
__device__ __forceinline__ bool tb_tile(const TbArgs &a, int b, int tx, int ty, const TbStart &t,
                                        uint32_t bar, uint32_t parity, float4 *tb_smem,
                                        double &wsum) {
    constexpr int RW = TW + 2 * K, RH = TH + 2 * K, RN = RW * RH;
    float4 *sP = tb_smem;                                  // RN
    float4 *sWR = sP + RN;                                 // RN
    float2 *sU = reinterpret_cast<float2 *>(sWR + RN);     // RN
    const int nx = a.nx, ny = a.ny;
    const size_t off = (size_t)b * a.stride;
    const int cur = t.cur, kk = t.kk;
    // accepted state in, final state to the other of buffers 0/1, snapshots
    // after iterations 1..K-1 to the snapshot set not containing the input
    const int fin = cur == 0 ? 1 : 0;
    const int snap = (cur >= 2 && cur < 2 + (K - 1)) ? 2 + (K - 1) : 2;
    const float2 *__restrict__ Uin = state_buf(a.U0, a.U1, cur) + off;
    float2 *__restrict__ Uout = state_buf(a.U0, a.U1, fin) + off;
    const float4 *__restrict__ Pin = state_buf(a.P0, a.P1, cur) + off;
    float4 *__restrict__ Pout = state_buf(a.P0, a.P1, fin) + off;
    const float4 *__restrict__ Wg = a.WR + off;
    const int ox = tx * TW - K, oy = ty * TH - K;
    const bool interior = ox >= 1 && oy >= 1 && ox + RW <= nx - 1 && oy + RH <= ny - 1;

    // the region: three TMA boxes (zero outside the level) completing on one
    // mbarrier, or plain loads where no tensor maps describe the level
    const uint32_t sbase = smem_u32(tb_smem);
    if (a.use_tma && (sbase & 127u) == 0) {
        if (threadIdx.x == 0) {
            mbar_arrive_expect_tx(bar, (uint32_t)RN * 40u);
            tma_load_4d(sbase, &a.tmP, 2 * ox, oy, b, cur, bar);
            tma_load_3d(sbase + RN * 16, &a.tmW, 2 * ox, oy, b, bar);
            tma_load_4d(sbase + RN * 32, &a.tmU, ox, oy, b, cur, bar);
        }
        const bool ok = mbar_wait_bounded(bar, parity);
        if (__syncthreads_or(!ok)) {
            // give up this tile: report, let the copies land (bounded), leave
            // without arriving (the host treats the plan's results as lost)
            if (threadIdx.x == 0) atomicExch(a.err, 1);
            mbar_wait_bounded(bar, parity);
            return false;
        }
    } else {
        for (int i = threadIdx.x; i < RN; i += NT) {
            const int x = ox + i % RW, y = oy + i / RW;
            float4 p = make_float4(0.f, 0.f, 0.f, 0.f), w = p;
            float2 u = make_float2(0.f, 0.f);
            if (x >= 0 && x < nx && y >= 0 && y < ny) {
                const size_t q = (size_t)y * nx + x;
                p = __ldcg(Pin + q);
                w = Wg[q];
                u = __ldcg(Uin + q);
            }
            sP[i] = p;
            sWR[i] = w;
            sU[i] = u;
        }
        __syncthreads();
    }

    // the owned tile is exact after every iteration: store it
    auto store_owned = [&](float2 *__restrict__ Ud, float4 *__restrict__ Pd) {
        for (int i = threadIdx.x; i < TW * TH; i += NT) {
            const int tx2 = i % TW, ty2 = i / TW;
            const int x = ox + K + tx2, y = oy + K + ty2;
            if (x >= nx || y >= ny) continue;
            const int r = (ty2 + K) * RW + tx2 + K;
            const size_t q = (size_t)y * nx + x;
            Ud[q] = sU[r];
            Pd[q] = sP[r];
        }
    };
    wsum = 0.0;
#pragma unroll
    for (int j = 0; j < K; j++) {
        if (j < kk) {  // uniform over the block
            double e = 0.0;
            if (interior)
                tb_iteration<TW, TH, K, NT, true>(j + 1, sP, sWR, sU, ox, oy, nx, ny, a.l_t,
                                                  a.theta, a.taut, e);
            else
                tb_iteration<TW, TH, K, NT, false>(j + 1, sP, sWR, sU, ox, oy, nx, ny, a.l_t,
                                                   a.theta, a.taut, e);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
            e = __shfl_sync(0xffffffffu, e, 0);
            if ((threadIdx.x & 31) == j) wsum = e;
            if (t.snaps && j + 1 < kk) {  // snapshot: the state a stop after iteration j+1 accepts
                store_owned(state_buf(a.U0, a.U1, snap + j) + off, state_buf(a.P0, a.P1, snap + j) + off);
                // the next iteration updates u and p in place: every thread must
                // have read its share of the snapshot first
                __syncthreads();
            }
        }
    }
    store_owned(Uout, Pout);
    return true;
}

template <int TW, int TH, int K, int NT>
__global__ void __launch_bounds__(NT, tb_min_blocks(NT)) k_tvl1_tb(const __grid_constant__ TbArgs a) {
    extern __shared__ __align__(128) float4 tb_smem[];
    __shared__ __align__(8) unsigned long long s_bar;
    const int b = blockIdx.z;
    TvCtrl *ctrl = a.ctrl + b;
    // The pair's control block changes in this launch only once all of the
    // pair's blocks have read it (the last to arrive writes it), so the reads
    // may be served from L1: blocks after the first on an SM, and the blocks of
    // a pair that already stopped, leave without a trip to L2.
    if (__ldca(&ctrl->stop)) return;
    TbStart t;
    t.cur = __ldca(&ctrl->cur);
    t.n0 = __ldca(&ctrl->n);
    t.redo = __ldca(&ctrl->redo);
    t.kk = t.redo > 0 ? t.redo : imin(K, a.max_it - t.n0);
    // block-uniform: every block of the pair reads the same control block
    t.snaps = false;
    if (t.redo == 0) {
        const float q = fminf(__ldca(&ctrl->decay), 1.0f);
        float qk = 1.0f;
#pragma unroll
        for (int j = 1; j < K; j++) qk *= q;
        t.snaps = __ldca(&ctrl->last_err) * qk < kSnapMargin * a.eps2;
    }
    const uint32_t bar = smem_u32(&s_bar);
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    __syncthreads();  // the barrier is initialised before anyone waits on it
    double wsum;
    if (!tb_tile<TW, TH, K, NT>(a, b, blockIdx.x, blockIdx.y, t, bar, 0, tb_smem, wsum)) return;
    const int fin = t.cur == 0 ? 1 : 0;
    const int snap = (t.cur >= 2 && t.cur < 2 + (K - 1)) ? 2 + (K - 1) : 2;
    tb_decide<K, NT>(a, ctrl, b, blockIdx.y * gridDim.x + blockIdx.x, gridDim.x * gridDim.y, wsum,
                     t.kk, fin, t.snaps ? snap : -1, t.redo, t.n0, nullptr, nullptr,
                     reinterpret_cast<double *>(tb_smem));
}

// Persistent form of k_tvl1_tb: one launch runs a whole warp stage of every
// pair.  Resident blocks take (pair, tile) items from a device work queue:
// each pair hands out the T tiles of its current block of K iterations; the
// last tile to finish takes the pair's stopping decision (tb_decide) and
// either stops the pair or opens its next block of iterations.  A block
// without work looks at the other pairs, so while one pair waits for the last
// tiles of a block of iterations the others fill the SMs, and no launch runs
// after a pair stopped.  Every item is exactly one k_tvl1_tb block (same
// tiles, iterations, decisions and bits).  No block waits while it holds an
// item, so items always finish; a block with nothing to take sleeps briefly,
// and gives up with the error flag after kWaitNs without finding work.
template <int TW, int TH, int K, int NT>
__global__ void __launch_bounds__(NT, tb_min_blocks(NT)) k_tvl1_q(const __grid_constant__ TbArgs a, TbQueue *q,
                                                  int *left, int tiles_x, int ntiles, int B) {
    extern __shared__ __align__(128) float4 tb_smem[];
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ int s_b, s_tile;
    // thread 0 only (in shared memory, not in every thread's registers): the
    // pair last worked on (first pair to look at), and a tile of that pair's
    // current block of iterations claimed ahead
    __shared__ int s_hint, s_ahead;
    __shared__ TbStart s_t;
    const uint32_t bar = smem_u32(&s_bar);
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
        s_hint = blockIdx.x % B;
        s_ahead = -1;
    }
    uint32_t parity = 0;
    for (;;) {
        if (threadIdx.x == 0) {
            int hint = s_hint, ahead = s_ahead;
            int got_b = -1, got_t = 0;
            if (ahead >= 0) {
                // claimed while this block held a tile of the same block of
                // iterations, which therefore had not been decided: the start
                // state in s_t still holds
                got_b = hint;
                got_t = ahead;
                ahead = -1;
            } else {
                unsigned long long t0 = 0;
                for (;;) {
                    for (int k = 0; k < B && got_b < 0; k++) {
                        const int bb = hint + k < B ? hint + k : hint + k - B;
                        if (*((volatile int *)&a.ctrl[bb].stop)) continue;
                        if (*((volatile unsigned long long *)&q[bb].ticket) >=
                            (unsigned long long)ntiles)
                            continue;
                        const unsigned long long tk = atomicAdd(&q[bb].ticket, 1ull);
                        if (tk < (unsigned long long)ntiles) {
                            got_b = bb;
                            got_t = (int)tk;
                        }
                    }
                    if (got_b >= 0 || *((volatile int *)left) <= 0) break;
                    if (t0 == 0) {
                        t0 = globaltimer();
                    } else if (globaltimer() - t0 > kWaitNs) {
                        atomicExch(a.err, 1);  // no work for kWaitNs: give up
                        break;
                    }
                    __nanosleep(256);
                }
                if (got_b >= 0) {
                    __threadfence();  // the pair's decision and state before its tiles are read
                    s_t = tb_start<K>(a, a.ctrl + got_b);
                    hint = got_b;
                }
            }
            if (got_b >= 0) {
                // generic-proxy writes of other blocks, then this block's TMA reads
                asm volatile("fence.proxy.async.global;\n" ::: "memory");
                fence_async_smem();  // this block's reads of the last region, then TMA writes
                // Claim the pair's next tile now; the answer is needed only
                // after this tile, so the atomic's latency is hidden.  Not
                // near the end of a block of iterations, where a tile claimed
                // by a busy block would wait for it while others are idle.
                if (got_t + 32 < ntiles) {
                    const unsigned long long tk = atomicAdd(&q[got_b].ticket, 1ull);
                    ahead = tk < (unsigned long long)ntiles ? (int)tk : -1;
                }
            }
            s_b = got_b;
            s_tile = got_t;
            s_hint = hint;
            s_ahead = ahead;
        }
        __syncthreads();
        const int b = s_b;
        if (b < 0) return;
        const TbStart t = s_t;
        const int tile = s_tile;
        double wsum;
        if (!tb_tile<TW, TH, K, NT>(a, b, tile % tiles_x, tile / tiles_x, t, bar, parity, tb_smem,
                                    wsum))
            return;
        parity ^= 1u;
        // The tile's stores reach other SMs before the pair's decision opens
        // its next block of iterations: the block barrier in tb_decide, then
        // thread 0's device-scope fence before it arrives (the pattern of a
        // grid-wide barrier).
        const int fin = t.cur == 0 ? 1 : 0;
        const int snap = (t.cur >= 2 && t.cur < 2 + (K - 1)) ? 2 + (K - 1) : 2;
        tb_decide<K, NT>(a, a.ctrl + b, b, tile, ntiles, wsum, t.kk, fin, t.snaps ? snap : -1,
                         t.redo, t.n0, q, left, reinterpret_cast<double *>(tb_smem));
        __syncthreads();  // shared state of this item is dead before the next claim
    }
}

// ---------------------------------------------------------------- whole level per block
// A level small enough for shared memory (u and p, 24 B per pixel) runs a
// whole warp stage in one launch: one block per pair, the inner iterations one
// after another separated by block barriers, the squared change of each
// summed in the block (per-thread double, fixed tree) and the stopping rule
// (tvl1.cpp:216) applied after each iteration.  No halo is recomputed and the
// state never leaves shared memory between iterations; I1wx, I1wy and rho_c
// come through the cache.  The per-pixel arithmetic is th_u_update and
// dual_update, as in the tiled kernels.
__global__ void __launch_bounds__(kLvNT) k_tvl1_level(TbArgs a) {
    extern __shared__ float4 lv_smem[];
    __shared__ double sred[kLvNT / 32];
    __shared__ int s_stop;
    const int nx = a.nx, ny = a.ny, N = nx * ny;
    float4 *sP = lv_smem;
    float2 *sU = reinterpret_cast<float2 *>(sP + N);
    const int b = blockIdx.x, tid = threadIdx.x;
    TvCtrl *ctrl = a.ctrl + b;
    const int cur = ctrl->cur;
    const int fin = cur == 0 ? 1 : 0;
    const size_t off = (size_t)b * a.stride;
    const float2 *__restrict__ Uin = state_buf(a.U0, a.U1, cur) + off;
    const float4 *__restrict__ Pin = state_buf(a.P0, a.P1, cur) + off;
    float2 *__restrict__ Uout = state_buf(a.U0, a.U1, fin) + off;
    float4 *__restrict__ Pout = state_buf(a.P0, a.P1, fin) + off;
    const float4 *__restrict__ Wg = a.WR + off;
    for (int i = tid; i < N; i += kLvNT) {
        sU[i] = Uin[i];
        sP[i] = Pin[i];
    }
    __syncthreads();
    int n = ctrl->n;
    bool done = n >= a.max_it;
    while (!done) {
        // TH + u update; only the pixel's own u is read, so in place
        double err = 0.0;
        for (int i = tid; i < N; i += kLvNT) {
            const int y = i / nx, x = i - y * nx;
            const float2 u = sU[i];
            const float4 pc = sP[i];
            const float4 pl = x > 0 ? sP[i - 1] : pc;   // unused on the left border
            const float4 pu = y > 0 ? sP[i - nx] : pc;  // unused on the top border
            const float2 un = th_u_update(u, __ldg(Wg + i), pc, pl, pu, x == 0,
                                          x == nx - 1, y == 0, y == ny - 1, a.l_t, a.theta);
            sU[i] = un;
            const float e1 = un.x - u.x, e2 = un.y - u.y;
            const float term = e1 * e1 + e2 * e2;
            err += (double)term;
        }
        __syncthreads();
        // dual update; only the pixel's own p is read, so in place
        for (int i = tid; i < N; i += kLvNT) {
            const int y = i / nx, x = i - y * nx;
            const float2 uc = sU[i];
            float f1x = 0.0f, f2x = 0.0f, f1y = 0.0f, f2y = 0.0f;
            if (x < nx - 1) {
                const float2 ur = sU[i + 1];
                f1x = ur.x - uc.x;
                f2x = ur.y - uc.y;
            }
            if (y < ny - 1) {
                const float2 ud = sU[i + nx];
                f1y = ud.x - uc.x;
                f2y = ud.y - uc.y;
            }
            sP[i] = dual_update(sP[i], f1x, f1y, f2x, f2y, a.taut);
        }
        const double tot = block_sum_double<kLvNT>(err, sred);  // barrier inside
        n++;
        if (tid == 0) {
            float e = (float)tot;
            e = e / (float)(nx * ny);
            s_stop = !(e > a.eps2) || n >= a.max_it;
        }
        __syncthreads();
        done = s_stop != 0;
    }
    for (int i = tid; i < N; i += kLvNT) {
        Uout[i] = sU[i];
        Pout[i] = sP[i];
    }
    if (tid == 0) {
        ctrl->n = n;
        ctrl->cur = fin;
        ctrl->stop = 1;
        a.iters[(size_t)b * a.iter_stride + a.stage] = n;
    }
}

// ---------------------------------------------------------------- level per cluster
// A level split into row bands over a cluster of kClC blocks, one cluster per
// pair: for levels that one block runs too slowly and tiles leave most SMs
// idle.  Each block keeps its band's u, p and warp data in shared memory and reads the one
// neighbouring row it needs -- p of the row above its band, u of the row below
// it -- from the adjacent block's shared memory (distributed shared memory).
// Per inner iteration the cluster synchronises twice: after the TH step and u
// update (u new everywhere, the bands' squared-change sums posted) and after
// the dual update (p new everywhere).  Every block adds the bands' sums in rank
// order from the others' shared memory, so all take the same stopping decision
// (tvl1.cpp:216) and run the same number of cluster barriers.  The per-pixel
// arithmetic is th_u_update and dual_update, as in the tiled kernels.
// (ly, x) of pixel i + NT from that of pixel i in rows of nx pixels.
template <int NT>
__device__ __forceinline__ void cl_step(int &ly, int &x, int nx) {
    ly += NT / nx;
    x += NT % nx;
    if (x >= nx) {
        x -= nx;
        ly += 1;
    }
}

template <int NT>
__global__ void __cluster_dims__(kClC, 1, 1) __launch_bounds__(NT) k_tvl1_cluster(TbArgs a) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const int c = (int)cluster.block_rank();
    extern __shared__ float4 cl_smem[];
    __shared__ double sred[NT / 32];
    __shared__ double s_part;
    const int nx = a.nx, ny = a.ny, tid = threadIdx.x;
    const int r0 = c * ny / kClC, r1 = (c + 1) * ny / kClC, nb = r1 - r0;
    const size_t cap = (size_t)cl_band_rows(ny) * nx;
    float4 *sP = cl_smem;
    float4 *sW = sP + cap;
    float2 *sU = reinterpret_cast<float2 *>(sW + cap);
    const int b = blockIdx.y;
    TvCtrl *ctrl = a.ctrl + b;
    const int cur = *((volatile int *)&ctrl->cur);
    const int fin = cur == 0 ? 1 : 0;
    const size_t off = (size_t)b * a.stride;
    const float2 *__restrict__ Uin = state_buf(a.U0, a.U1, cur) + off + (size_t)r0 * nx;
    const float4 *__restrict__ Pin = state_buf(a.P0, a.P1, cur) + off + (size_t)r0 * nx;
    const float4 *__restrict__ Wg = a.WR + off + (size_t)r0 * nx;
    const int N = nb * nx;
    for (int i = tid; i < N; i += NT) {
        sU[i] = Uin[i];
        sP[i] = Pin[i];
        sW[i] = Wg[i];
    }
    // the neighbours' rows: p of the band above (its last row), u of the band below (its first)
    const int nb_up = c > 0 ? r0 - (c - 1) * ny / kClC : 0;
    const float4 *upP = c > 0 ? cluster.map_shared_rank(sP, c - 1) + (size_t)(nb_up - 1) * nx : nullptr;
    const float2 *dnU = c + 1 < kClC ? cluster.map_shared_rank(sU, c + 1) : nullptr;
    cluster.sync();
    int n = *((volatile int *)&ctrl->n);
    bool done = n >= a.max_it;
    const int ly0 = tid / nx, x0 = tid - ly0 * nx;  // band row and column of pixel tid
    while (!done) {
        double err = 0.0;
        for (int i = tid, ly = ly0, x = x0; i < N; i += NT, cl_step<NT>(ly, x, nx)) {
            const int y = r0 + ly;
            const float2 u = sU[i];
            const float4 pc = sP[i];
            const float4 pl = x > 0 ? sP[i - 1] : pc;  // unused on the left border
            const float4 pu = y == 0 ? pc : (ly > 0 ? sP[i - nx] : upP[x]);  // unused on the top border
            const float2 un = th_u_update(u, sW[i], pc, pl, pu, x == 0, x == nx - 1, y == 0,
                                          y == ny - 1, a.l_t, a.theta);
            sU[i] = un;
            const float e1 = un.x - u.x, e2 = un.y - u.y;
            const float term = e1 * e1 + e2 * e2;
            err += (double)term;
        }
        const double bs = block_sum_double<NT>(err, sred);
        if (tid == 0) s_part = bs;
        cluster.sync();  // u new in every band, the bands' sums posted
        double tot = 0.0;
#pragma unroll
        for (int k = 0; k < kClC; k++) tot += *cluster.map_shared_rank(&s_part, k);
        n++;
        float e = (float)tot;
        e = e / (float)(nx * ny);
        const bool stop = !(e > a.eps2) || n >= a.max_it;
        for (int i = tid, ly = ly0, x = x0; i < N; i += NT, cl_step<NT>(ly, x, nx)) {
            const int y = r0 + ly;
            const float2 uc = sU[i];
            float f1x = 0.0f, f2x = 0.0f, f1y = 0.0f, f2y = 0.0f;
            if (x < nx - 1) {
                const float2 ur = sU[i + 1];
                f1x = ur.x - uc.x;
                f2x = ur.y - uc.y;
            }
            if (y < ny - 1) {
                const float2 ud = ly + 1 < nb ? sU[i + nx] : dnU[x];
                f1y = ud.x - uc.x;
                f2y = ud.y - uc.y;
            }
            sP[i] = dual_update(sP[i], f1x, f1y, f2x, f2y, a.taut);
        }
        cluster.sync();  // p new in every band; the sums may be overwritten
        done = stop;
    }
    float2 *__restrict__ Uout = state_buf(a.U0, a.U1, fin) + off + (size_t)r0 * nx;
    float4 *__restrict__ Pout = state_buf(a.P0, a.P1, fin) + off + (size_t)r0 * nx;
    for (int i = tid; i < N; i += NT) {
        Uout[i] = sU[i];
        Pout[i] = sP[i];
    }
    if (c == 0 && tid == 0) {
        ctrl->n = n;
        ctrl->cur = fin;
        ctrl->stop = 1;
        a.iters[(size_t)b * a.iter_stride + a.stage] = n;
    }
}

// ---------------------------------------------------------------- energy
// E = sum |grad u1| + |grad u2| (forward differences, double) + lambda *
// sum |rho(u)| with rho linearised at the current warp.  Last block of a pair
// writes ctrl.energy and, if slot >= 0, energy_out[b * slots + slot].
constexpr int kEnNT = 256;
__global__ void __launch_bounds__(kEnNT) k_energy(const float4 *WR, const float2 *U0,
                                                  const float2 *U1, size_t stride, int nx,
                                                  int ny, float lambda, TvCtrl *ctrl,
                                                  double *partials, int max_blocks,
                                                  double *energy_out, int slots, int slot,
                                                  int expect_n) {
    const int b = blockIdx.y;
    const size_t off = (size_t)b * stride;
    const float2 *U = state_buf(U0, U1, ctrl[b].cur) + off;
    const int N = nx * ny;
    double tv = 0.0, data = 0.0;
    for (int i = blockIdx.x * kEnNT + threadIdx.x; i < N; i += gridDim.x * kEnNT) {
        const int x = i % nx, y = i / nx;
        const float2 uc = U[i];
        double f1x = 0, f1y = 0, f2x = 0, f2y = 0;
        if (x < nx - 1) { const float2 r = U[i + 1]; f1x = (double)(r.x - uc.x); f2x = (double)(r.y - uc.y); }
        if (y < ny - 1) { const float2 d = U[i + nx]; f1y = (double)(d.x - uc.x); f2y = (double)(d.y - uc.y); }
        tv += sqrt(f1x * f1x + f1y * f1y) + sqrt(f2x * f2x + f2y * f2y);
        const float4 w = WR[off + i];
        const float rho = w.z + (w.x * uc.x + w.y * uc.y);
        data += fabs((double)rho);
    }
    __shared__ double sred[kEnNT / 32];
    __shared__ int s_last;
    const double s = block_sum_double<kEnNT>(tv + (double)lambda * data, sred);
    double *part = partials + (size_t)b * max_blocks;
    if (threadIdx.x == 0) {
        part[blockIdx.x] = s;
        __threadfence();
        const unsigned prev = atomicAdd(&ctrl[b].arrive, 1u);
        s_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double acc = 0.0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += kEnNT) acc += __ldcg(part + k);
    const double tot = block_sum_double<kEnNT>(acc, sred);
    if (threadIdx.x == 0) {
        ctrl[b].energy = tot;
        // a trace slot is written only if iteration `expect_n` really ran
        if (slot >= 0 && (expect_n < 0 || ctrl[b].n == expect_n))
            energy_out[(size_t)b * slots + slot] = tot;
        ctrl[b].arrive = 0;
    }
}

// Non-linearised TV-L1 energy of (u1, u2) at the finest scale: sum of
// |grad u1| + |grad u2| (forward differences, double) + lambda * sum
// |I1(x+u) - I0(x)| with the bicubic sample and border zeroing of the warp
// (bicubic_interpolation.cpp:141-163).  Used to compare two solutions of the
// same pair at the same linearisation-free cost.
__global__ void __launch_bounds__(kEnNT) k_energy_true(const float *__restrict__ pyr, size_t lp,
                                                       const float2 *U0, const float2 *U1,
                                                       size_t stride, int nx, int ny,
                                                       float lambda, const TvCtrl *ctrl,
                                                       double *partials, int max_blocks,
                                                       unsigned *arrive, double *out) {
    const int b = blockIdx.y;
    const float2 *U = state_buf(U0, U1, ctrl[b].cur) + (size_t)b * stride;
    const float *I0 = pyr + (size_t)(2 * b) * lp;
    const float *I1 = pyr + (size_t)(2 * b + 1) * lp;
    const int N = nx * ny;
    double acc = 0.0;
    for (int i = blockIdx.x * kEnNT + threadIdx.x; i < N; i += gridDim.x * kEnNT) {
        const int x = i % nx, y = i / nx;
        const float2 uc = U[i];
        double f1x = 0, f1y = 0, f2x = 0, f2y = 0;
        if (x < nx - 1) { const float2 r = U[i + 1]; f1x = (double)(r.x - uc.x); f2x = (double)(r.y - uc.y); }
        if (y < ny - 1) { const float2 d = U[i + nx]; f1y = (double)(d.x - uc.x); f2y = (double)(d.y - uc.y); }
        const float w = bicubic_at(I1, (float)x + uc.x, (float)y + uc.y, nx, ny, true);
        acc += sqrt(f1x * f1x + f1y * f1y) + sqrt(f2x * f2x + f2y * f2y) +
               (double)lambda * fabs((double)(w - __ldg(I0 + i)));
    }
    __shared__ double sred[kEnNT / 32];
    __shared__ int s_last;
    const double s = block_sum_double<kEnNT>(acc, sred);
    double *part = partials + (size_t)b * max_blocks;
    if (threadIdx.x == 0) {
        part[blockIdx.x] = s;
        __threadfence();
        s_last = (atomicAdd(arrive + b, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double a2 = 0.0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += kEnNT) a2 += __ldcg(part + k);
    const double tot = block_sum_double<kEnNT>(a2, sred);
    if (threadIdx.x == 0) {
        out[b] = tot;
        arrive[b] = 0;
    }
}

// ---------------------------------------------------------------- output
// The accepted flow of pair b (blockIdx.z) into its output planes: the
// plan's own buffer or the caller's device planes (any row pitch).
__global__ void k_split(const float2 *U0, const float2 *U1, size_t stride, int w, int h,
                        const OutRef *__restrict__ outs, const TvCtrl *ctrl) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const int b = blockIdx.z;
    const float2 u = (state_buf(U0, U1, ctrl[b].cur) + (size_t)b * stride)[(size_t)y * w + x];
    const OutRef o = outs[b];
    o.u[(size_t)y * o.pitch + x] = u.x;
    o.v[(size_t)y * o.pitch + x] = u.y;
}

// ================================================================ launchers
GaussTaps make_zoom_taps(float zfactor) { return make_taps(zoom_sigma(zfactor)); }

void launch_gauss(const float *src, float *dst, int nx, int ny, size_t stride,
                  const GaussTaps &t, int planes, cudaStream_t st) {
    dim3 g(div_up(nx, kGaussTW), div_up(ny, kGaussTH), planes);
    if (t.size == 5)
        k_gauss<0, 4><<<g, kGaussNT, 0, st>>>(src, dst, nx, ny, stride, t, nullptr, 0, nullptr);
    else if (t.size == 6)
        k_gauss<0, 5><<<g, kGaussNT, 0, st>>>(src, dst, nx, ny, stride, t, nullptr, 0, nullptr);
    else
        k_gauss<0, 0><<<g, kGaussNT, 0, st>>>(src, dst, nx, ny, stride, t, nullptr, 0, nullptr);
}

void launch_resample(const float *src, size_t sstride, int nx, int ny, float *dst,
                     size_t dstride, int nxx, int nyy, float dx, float dy, int planes,
                     cudaStream_t st) {
    dim3 blk(32, 8), g(div_up(nxx, 32), div_up(nyy, 8), planes);
    k_resample<<<g, blk, 0, st>>>(src, sstride, nx, ny, dst, dstride, nxx, nyy, dx, dy);
}

int launch_zoom_out(const float *src, size_t sstride, int nx, int ny, float *T, float *dst,
                    size_t dstride, int nxx, int nyy, float zfactor, const GaussTaps &t,
                    int planes, cudaStream_t st) {
    if (zfactor == 0.5f && t.size - 1 <= kDecMaxR) {
        dim3 g(div_up(nxx, kDecTW), div_up(nyy, kDecTH), planes);
        if (t.size == 6)  // sigma 0.6 sqrt(3) of zfactor 1/2: radius 5
            k_gauss_dec2<5><<<g, kDecNT, 0, st>>>(src, sstride, nx, ny, dst, dstride, nxx, nyy, t);
        else
            k_gauss_dec2<0><<<g, kDecNT, 0, st>>>(src, sstride, nx, ny, dst, dstride, nxx, nyy, t);
        return 1;
    }
    launch_gauss(src, T, nx, ny, sstride, t, planes, st);
    launch_resample(T, sstride, nx, ny, dst, dstride, nxx, nyy, zfactor, zfactor, planes, st);
    return 2;
}

// ================================================================ host plan
// cuTensorMapEncodeTiled, looked up in the driver once (null if unavailable).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// A tiled map of 8-byte elements, zero fill outside; dims innermost first,
// byte strides of dims 1..rank-1.
bool encode_map8(CUtensorMap *m, void *base, int rank, const cuuint64_t *dims,
                 const cuuint64_t *strides, const cuuint32_t *box) {
    const PFN_cuTensorMapEncodeTiled_v12000 fn = tensor_map_encoder();
    if (!fn) return false;
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, (cuuint32_t)rank, base, dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor maps of k_tvl1_tb's region loads for tile configuration cfg on a
// level of nx x ny (planes of N0 elements, B pairs, kStateBufs buffers of u
// and p).  TMA wants 16-byte row and plane strides, so u (8 bytes a pixel)
// needs even nx and N0; otherwise the kernel loads the region itself.
static void tb_maps(TbArgs &ta, int cfg, int nx, int ny, int B, size_t N0, float4 *P0, float2 *U0,
                    const float4 *WR, int *err) {
    ta.use_tma = 0;
    ta.err = err;
    if (cfg >= kTbNumCfgs || (nx & 1) || (N0 & 1)) return;
    const cuuint32_t rw = (cuuint32_t)(kTbCfgs[cfg].tw + 2 * kTbK), rh = (cuuint32_t)(kTbCfgs[cfg].th + 2 * kTbK);
    const cuuint64_t X = (cuuint64_t)nx, Y = (cuuint64_t)ny, NB = (cuuint64_t)B, N = N0;
    const cuuint64_t dp[4] = {2 * X, Y, NB, (cuuint64_t)kStateBufs}, sp[3] = {16 * X, 16 * N, 16 * N * NB};
    const cuuint32_t bp[4] = {2 * rw, rh, 1, 1};
    const cuuint64_t du[4] = {X, Y, NB, (cuuint64_t)kStateBufs}, su[3] = {8 * X, 8 * N, 8 * N * NB};
    const cuuint32_t bu[4] = {rw, rh, 1, 1};
    const cuuint64_t dw[3] = {2 * X, Y, NB}, sw[2] = {16 * X, 16 * N};
    const cuuint32_t bw[3] = {2 * rw, rh, 1};
    ta.use_tma = encode_map8(&ta.tmP, P0, 4, dp, sp, bp) && encode_map8(&ta.tmU, U0, 4, du, su, bu) &&
                 encode_map8(&ta.tmW, const_cast<float4 *>(WR), 3, dw, sw, bw);
}

// A plan needs no repair after a timeout: every warp stage starts with
// k_warp re-arming each pair's control block and work queue, so the next
// call runs from a clean state (tested with OFLOW_INJECT_TIMEOUT).
void TvPlan::check_device_error() {
    if (err_.take())
        throw Error(OFLOW_ERR_TIMEOUT,
                    "tvl1: a bounded device wait gave up (a tile's TMA load or the work queue)");
}

template <int TW, int TH, int NT>
static void tb_launch(dim3 g, cudaStream_t st, const TbArgs &ta) {
    k_tvl1_tb<TW, TH, kTbK, NT><<<g, NT, tb_smem_bytes(TW, TH), st>>>(ta);
}

static void tb_launch_cfg(int cfg, dim3 g, cudaStream_t st, const TbArgs &ta) {
    if (cfg == kClusterCfg) {
        // 256 threads where they cover a band in one pass, else 512 (1024
        // threads leave one block per SM: 32 clusters of 8 then take two
        // waves, and the 128x55 level took 1.6 ms instead of 0.95)
        const int band = cl_band_rows(ta.ny) * ta.nx;
        const size_t smem = (size_t)band * (2 * sizeof(float4) + sizeof(float2));
        if (band <= 256)
            k_tvl1_cluster<256><<<dim3(kClC, g.z), 256, smem, st>>>(ta);
        else
            k_tvl1_cluster<512><<<dim3(kClC, g.z), 512, smem, st>>>(ta);
        return;
    }
    if (cfg == kLevelCfg) {
        const size_t smem = (size_t)ta.nx * ta.ny * (sizeof(float4) + sizeof(float2));
        k_tvl1_level<<<g.z, kLvNT, smem, st>>>(ta);
        return;
    }
    switch (cfg) {
        case 0: tb_launch<64, 32, 512>(g, st, ta); break;
        case 1: tb_launch<64, 16, 256>(g, st, ta); break;
        case 2: tb_launch<32, 16, 256>(g, st, ta); break;
        default: tb_launch<16, 8, 128>(g, st, ta); break;
    }
}

// Resident blocks of the persistent kernel per SM, for each tile shape.
template <int TW, int TH, int NT>
static int tb_queue_occupancy() {
    static int occ = -1;
    if (occ < 0) {
        int n = 0;
        OF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_tvl1_q<TW, TH, kTbK, NT>, NT,
                                                              tb_smem_bytes(TW, TH)));
        occ = imax(n, 1);
    }
    return occ;
}

template <int TW, int TH, int NT>
static void tb_launch_q(dim3 g, cudaStream_t st, const TbArgs &ta, TbQueue *q, int *left,
                        int share) {
    const int ntiles = (int)(g.x * g.y);
    const int slots = imax(1, tb_queue_occupancy<TW, TH, NT>() * kNumSMs / imax(share, 1));
    const int blocks = imin(ntiles * (int)g.z, slots);
    k_tvl1_q<TW, TH, kTbK, NT><<<blocks, NT, tb_smem_bytes(TW, TH), st>>>(ta, q, left, (int)g.x,
                                                                         ntiles, (int)g.z);
}

// A whole tiled warp stage as one persistent launch (k_tvl1_q).
// share > 1: the plan runs beside share - 1 others of its kind (the chunks of
// a host batch) and takes that fraction of the resident slots.
static void tb_launch_queue(int cfg, dim3 g, cudaStream_t st, const TbArgs &ta_in, TbQueue *q,
                            int *left, int predict, int share) {
    TbArgs ta = ta_in;
    ta.predict = predict;
    switch (cfg) {
        case 0: tb_launch_q<64, 32, 512>(g, st, ta, q, left, share); break;
        case 1: tb_launch_q<64, 16, 256>(g, st, ta, q, left, share); break;
        case 2: tb_launch_q<32, 16, 256>(g, st, ta, q, left, share); break;
        default: tb_launch_q<16, 8, 128>(g, st, ta, q, left, share); break;
    }
}

static void tb_set_smem_attrs() {
    OF_CUDA(cudaFuncSetAttribute(k_tvl1_q<64, 32, kTbK, 512>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tb_smem_bytes(64, 32)));
    OF_CUDA(cudaFuncSetAttribute(k_tvl1_q<64, 16, kTbK, 256>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tb_smem_bytes(64, 16)));
    OF_CUDA(cudaFuncSetAttribute(k_tvl1_tb<64, 32, kTbK, 512>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tb_smem_bytes(64, 32)));
    OF_CUDA(cudaFuncSetAttribute(k_tvl1_tb<64, 16, kTbK, 256>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tb_smem_bytes(64, 16)));
    OF_CUDA(cudaFuncSetAttribute(k_tvl1_level, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kLvMaxPx * (int)(sizeof(float4) + sizeof(float2))));
    OF_CUDA(cudaFuncSetAttribute(k_tvl1_cluster<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kClMaxSmem));
    OF_CUDA(cudaFuncSetAttribute(k_tvl1_cluster<512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kClMaxSmem));
}

static int tb_tiles(int cfg, int nx, int ny) {
    int tw, th;
    if (!cfg_tile(cfg, tw, th)) return 1;
    return div_up(nx, tw) * div_up(ny, th);
}

static dim3 tb_grid(int cfg, int nx, int ny, int B) {
    int tw, th;
    if (!cfg_tile(cfg, tw, th)) return dim3(1, 1, B);
    return dim3(div_up(nx, tw), div_up(ny, th), B);
}

// Largest tile whose grid still gives every SM two blocks; small scales get
// small tiles (more blocks, shorter per-launch latency).  OFLOW_TB_CFG forces
// one configuration (used to time them against each other).
static int tb_pick(int nx, int ny, int B) {
    if (const char *e = getenv("OFLOW_TB_CFG")) {
        const int c = atoi(e);
        if (c >= 0 && c < kTbNumCfgs) return c;
        if (c == kLevelCfg && level_fits(nx, ny)) return c;
        if (c == kClusterCfg && cluster_fits(nx, ny)) return c;
    }
    if (level_fits(nx, ny)) return kLevelCfg;
    for (int c = 0; c < kTbNumCfgs; c++)
        if (tb_tiles(c, nx, ny) * B >= 2 * kNumSMs) return c;
    return kTbNumCfgs - 1;
}

// a configuration from a tuning table, if it is valid for this level
static bool cfg_valid(int c, int nx, int ny) {
    return (c >= 0 && c < kTbNumCfgs) || (c == kLevelCfg && level_fits(nx, ny)) ||
           (c == kClusterCfg && cluster_fits(nx, ny));
}

TvPlan::TvPlan(int w, int h, int B, int dtype, const oflow_tvl1_params &prm, bool trace,
               const TuneTable *tuned, int start_scale)
    : w_(w), h_(h), B_(B), dtype_(dtype), prm_(prm), trace_(trace) {
    OF_CHECK(w >= 8 && h >= 8, "tvl1: frames must be at least 8x8");
    OF_CHECK(B >= 1, "tvl1: empty batch");
    OF_CHECK(prm.zfactor > 0.0f && prm.zfactor < 1.0f, "tvl1: zfactor must be in (0,1)");
    OF_CHECK(prm.warps >= 1 && prm.warps <= OFLOW_MAX_WARPS, "tvl1: warps out of range");
    OF_CHECK(prm.max_iterations >= 0, "tvl1: max_iterations < 0");
    OF_CHECK(prm.theta > 0.0f, "tvl1: theta must be > 0");
    ns_ = tvl1_nscales(w, h, prm.nscales, prm.zfactor);
    OF_CHECK(ns_ >= 1 && ns_ <= OFLOW_MAX_SCALES, "tvl1: number of scales out of range");
    nx_[0] = w;
    ny_[0] = h;
    for (int s = 1; s < ns_; s++) tvl1_zoom_size(nx_[s - 1], ny_[s - 1], &nx_[s], &ny_[s], prm.zfactor);
    taps0_ = make_taps(0.8f);
    tapsz_ = make_taps(zoom_sigma(prm.zfactor));
    // every blurred level must hold the whole window (mask.cpp:231)
    OF_CHECK(taps0_.size <= w && taps0_.size <= h, "tvl1: frame smaller than the Gaussian window");
    for (int s = 0; s + 1 < ns_; s++)
        OF_CHECK(tapsz_.size <= nx_[s] && tapsz_.size <= ny_[s],
                 "tvl1: pyramid level smaller than the Gaussian window");
    for (int s = 0; s < ns_; s++) OF_CHECK(nx_[s] >= 2 && ny_[s] >= 2, "tvl1: level below 2x2");
    OF_CHECK(start_scale < ns_, "tvl1: warm-start scale beyond the pyramid");
    s0_ = start_scale >= 0 ? start_scale : ns_ - 1;
    warm_ = start_scale >= 0;
    for (int s = 0; s < OFLOW_MAX_SCALES; s++) {
        sw_[s] = prm.warps;
        si_[s] = prm.max_iterations;
    }

    const size_t N0 = (size_t)w * h;
    N0_ = N0;
    iter_blocks_ = div_up(w, kIterTW) * div_up(h, kIterTH);
    for (int s = 0; s < ns_; s++) {
        const auto it = tuned ? tuned->find(tune_key(nx_[s], ny_[s], B)) : TuneTable::const_iterator();
        tb_cfg_[s] = (tuned && it != tuned->end() && cfg_valid(it->second, nx_[s], ny_[s]))
                         ? it->second
                         : tb_pick(nx_[s], ny_[s], B);
        for (int c = 0; c < kNumIterCfgs; c++)  // any configuration may run while tuning
            iter_blocks_ = imax(iter_blocks_, tb_tiles(c, nx_[s], ny_[s]) * kTbK);
    }
    ingest_blocks_ = imin(div_up((int)N0, kIngestNT * kIngestPPT), 1024);
    energy_blocks_ = imin(div_up((int)N0, kEnNT * 4), 512);
    max_blocks_ = imax(iter_blocks_, energy_blocks_);
    pyr_off_[0] = 0;
    for (int s = 1; s < ns_; s++) pyr_off_[s] = pyr_off_[s - 1] + (size_t)2 * B * nx_[s - 1] * ny_[s - 1];
    const size_t pyr_total = pyr_off_[ns_ - 1] + (size_t)2 * B * nx_[ns_ - 1] * ny_[ns_ - 1];
    const size_t esz = dtype == OFLOW_U8 ? 1 : 4;

    o_raw_ = ar_.reserve(2 * B * N0 * esz);
    o_T_ = ar_.reserve(2 * B * N0 * 4);
    o_pyr_ = ar_.reserve(pyr_total * 4);
    o_cc_ = ar_.reserve(B * N0 * 72);  // WarpCoef: 3 x double2, float4, float2 per texel
    o_WR_ = ar_.reserve(B * N0 * 16);
    o_U0_ = ar_.reserve(kStateBufs * B * N0 * 8);  // buffer k at U0 + k*B*N0
    o_Uz_ = ar_.reserve(B * N0 * 8);
    o_P0_ = ar_.reserve(kStateBufs * B * N0 * 16);
    o_out_ = ar_.reserve(2 * B * N0 * 4);
    o_ctrl_ = ar_.reserve(B * sizeof(TvCtrl));
    o_part_ = ar_.reserve((size_t)B * max_blocks_ * 8);
    o_recs_ = ar_.reserve((size_t)B * ingest_blocks_ * 4 * sizeof(NormRec));
    iter_stride_ = ns_ * prm.warps;
    o_iters_ = ar_.reserve((size_t)B * iter_stride_ * 4);
    energy_slots_ = trace ? ns_ * prm.warps * prm.max_iterations : 1;
    o_energy_ = ar_.reserve((size_t)B * energy_slots_ * 8);
    o_tarr_ = ar_.reserve(sizeof(unsigned) * B);
    o_tout_ = ar_.reserve(sizeof(double) * B);
    o_frames_ = ar_.reserve(sizeof(FrameRef) * 2 * B);
    o_queue_ = ar_.reserve(sizeof(TbQueue) * B);
    o_left_ = ar_.reserve(sizeof(int));
    o_otab_ = ar_.reserve(sizeof(OutRef) * B);
    ar_.commit();
    frames_.resize(2 * (size_t)B);
    outs_.resize((size_t)B);
    for (int b = 0; b < B; b++) {
        for (int k = 0; k < 2; k++) bind_raw(b, k);
        bind_own_out(b);
    }
    OF_CUDA(cudaMemcpy(ar_.at<FrameRef>(o_frames_), frames_.data(), sizeof(FrameRef) * frames_.size(),
                       cudaMemcpyHostToDevice));
    OF_CUDA(cudaMemcpy(ar_.at<OutRef>(o_otab_), outs_.data(), sizeof(OutRef) * outs_.size(),
                       cudaMemcpyHostToDevice));
    OF_CUDA(cudaMemset(ar_.at<char>(o_ctrl_), 0, B * sizeof(TvCtrl)));
    OF_CUDA(cudaMemset(ar_.at<char>(o_queue_), 0, B * sizeof(TbQueue)));
    // OFLOW_TB_QUEUE=0 runs the tiled stages as one launch per block of K
    // iterations (k_tvl1_tb) instead of the persistent work queue (k_tvl1_q)
    if (const char *e = getenv("OFLOW_TB_QUEUE")) queue_off_env_ = atoi(e) == 0;
    queue_ = !queue_off_env_;
    // The queue form sizes each block of iterations to end at the stop its
    // error decay predicts and drops the snapshots of a shortened block (2,
    // the default; 1: keeps them; 0: full blocks)
    predict_ = 2;
    if (const char *e = getenv("OFLOW_TB_PREDICT")) predict_ = atoi(e);
    // scales above a warm start's first scale never record a count
    OF_CUDA(cudaMemset(ar_.at<char>(o_iters_), 0, (size_t)B * iter_stride_ * 4));
    tb_set_smem_attrs();
}

void TvPlan::bind_frame(int b, int k, const void *p, int pitch) {
    frames_[2 * (size_t)b + k] = FrameRef{p, pitch};
}
void TvPlan::bind_raw(int b, int k) { frames_[2 * (size_t)b + k] = FrameRef{raw_input(b, k), w_}; }
void TvPlan::bind_out(int b, float *u, float *v, int pitch) { outs_[b] = OutRef{u, v, pitch ? pitch : w_}; }
void TvPlan::bind_own_out(int b) {
    float *o = ar_.at<float>(o_out_);
    outs_[b] = OutRef{o + (size_t)b * N0_, o + (size_t)(B_ + b) * N0_, w_};
}
void TvPlan::upload_frames(cudaStream_t st) {
    // pageable sources: the runtime copies them out before returning
    OF_CUDA(cudaMemcpyAsync(ar_.at<FrameRef>(o_frames_), frames_.data(), sizeof(FrameRef) * frames_.size(),
                            cudaMemcpyHostToDevice, st));
    OF_CUDA(cudaMemcpyAsync(ar_.at<OutRef>(o_otab_), outs_.data(), sizeof(OutRef) * outs_.size(),
                            cudaMemcpyHostToDevice, st));
}
void TvPlan::run_eager(cudaStream_t st) {
    upload_frames(st);
    record(st);
}

void *TvPlan::raw_input(int b, int k) const {
    const size_t esz = dtype_ == OFLOW_U8 ? 1 : 4;
    return ar_.at<char>(o_raw_) + (size_t)(2 * b + k) * N0_ * esz;
}
float2 *TvPlan::ubuf(int k) const { return ar_.at<float2>(o_U0_) + (size_t)k * B_ * N0_; }
float4 *TvPlan::pbuf(int k) const { return ar_.at<float4>(o_P0_) + (size_t)k * B_ * N0_; }

const float *TvPlan::out_u(int b) const { return ar_.at<float>(o_out_) + (size_t)b * N0_; }
const float *TvPlan::out_v(int b) const { return ar_.at<float>(o_out_) + (size_t)(B_ + b) * N0_; }
const int *TvPlan::iters_dev() const { return ar_.at<int>(o_iters_); }
float2 *TvPlan::uz() const { return ar_.at<float2>(o_Uz_); }


void TvPlan::record(cudaStream_t st) {
    launches_ = 0;
    const int B = B_;
    const size_t N0 = N0_;
    float *T = ar_.at<float>(o_T_);
    float *pyr = ar_.at<float>(o_pyr_);
    WarpCoef wc;
    {
        const size_t n = (size_t)B * N0;
        wc.cc0 = ar_.at<double2>(o_cc_);
        wc.cc1 = wc.cc0 + n;
        wc.cc2 = wc.cc1 + n;
        wc.dv01 = reinterpret_cast<float4 *>(wc.cc2 + n);
        wc.dv2 = reinterpret_cast<float2 *>(wc.dv01 + n);
    }
    float4 *WR = ar_.at<float4>(o_WR_);
    float2 *U0 = ubuf(0), *U1 = ubuf(1), *Uz = ar_.at<float2>(o_Uz_);
    float4 *P0 = pbuf(0), *P1 = pbuf(1);
    TvCtrl *ctrl = ar_.at<TvCtrl>(o_ctrl_);
    double *part = ar_.at<double>(o_part_);
    NormRec *recs = ar_.at<NormRec>(o_recs_);
    int *iters = ar_.at<int>(o_iters_);
    double *energy = ar_.at<double>(o_energy_);
    TbQueue *queue = ar_.at<TbQueue>(o_queue_);
    int *left = ar_.at<int>(o_left_);
    // profile replays are captured: external event nodes keep timestamps;
    // each begin/end pair is tagged -1 (warp launch) or with its scale
    // (inner-iteration launch)
    auto mark_begin = [&](int tag) {
        if (!prof_) return;
        if (prof_->n_ev + 2 > (int)prof_->ev.size()) {
            cudaEvent_t e[2];
            OF_CUDA(cudaEventCreate(&e[0]));
            OF_CUDA(cudaEventCreate(&e[1]));
            prof_->ev.push_back(e[0]);
            prof_->ev.push_back(e[1]);
        }
        prof_->tag.push_back(tag);
        OF_CUDA(cudaEventRecordWithFlags(prof_->ev[prof_->n_ev++], st, cudaEventRecordExternal));
    };
    auto mark_end = [&]() {
        if (prof_)
            OF_CUDA(cudaEventRecordWithFlags(prof_->ev[prof_->n_ev++], st, cudaEventRecordExternal));
    };

    OF_CUDA(cudaMemsetAsync(iters, 0, sizeof(int) * (size_t)B * iter_stride_, st));
    // normalisation range of both frames, read through the frame table
    const FrameRef *frames = ar_.at<FrameRef>(o_frames_);
    {
        dim3 g(ingest_blocks_, B);
        if (dtype_ == OFLOW_U8)
            k_ingest<uint8_t><<<g, kIngestNT, 0, st>>>(frames, w_, h_, recs, ingest_blocks_);
        else
            k_ingest<float><<<g, kIngestNT, 0, st>>>(frames, w_, h_, recs, ingest_blocks_);
        k_norm_finalize<<<B, kNormNT, 0, st>>>(recs, ingest_blocks_, ctrl);
        launches_ += 2;
    }
    // conversion, normalisation and pre-smoothing of level 0 in one pass
    // (tvl1.cpp:137-144)
    {
        dim3 g(div_up(w_, kGaussTW), div_up(h_, kGaussTH), 2 * B);
        float *p0 = pyr + pyr_off_[0];
        const bool r4 = taps0_.size == 5;  // sigma 0.8: radius 4
        if (dtype_ == OFLOW_U8 && r4)
            k_gauss<1, 4><<<g, kGaussNT, 0, st>>>(nullptr, p0, w_, h_, N0, taps0_, ctrl, 1, frames);
        else if (dtype_ == OFLOW_U8)
            k_gauss<1, 0><<<g, kGaussNT, 0, st>>>(nullptr, p0, w_, h_, N0, taps0_, ctrl, 1, frames);
        else if (r4)
            k_gauss<2, 4><<<g, kGaussNT, 0, st>>>(nullptr, p0, w_, h_, N0, taps0_, ctrl, 1, frames);
        else
            k_gauss<2, 0><<<g, kGaussNT, 0, st>>>(nullptr, p0, w_, h_, N0, taps0_, ctrl, 1, frames);
        launches_ += 1;
    }
    // pyramid (tvl1.cpp:147-154)
    for (int s = 1; s < ns_; s++) {
        const int nx = nx_[s - 1], ny = ny_[s - 1];
        const size_t sp = (size_t)nx * ny, dp = (size_t)nx_[s] * ny_[s];
        launches_ += launch_zoom_out(pyr + pyr_off_[s - 1], sp, nx, ny, T, pyr + pyr_off_[s], dp,
                                     nx_[s], ny_[s], prm_.zfactor, tapsz_, 2 * B, st);
    }
    const float l_t = prm_.lambda * prm_.theta;
    const float taut = prm_.tau / prm_.theta;
    const float eps2 = prm_.epsilon * prm_.epsilon;
    const float inv = 1 / prm_.zfactor;
    for (int s = s0_; s >= 0; s--) {
        const int nx = nx_[s], ny = ny_[s];
        const size_t lp = (size_t)nx * ny;
        dim3 blk(32, 8), gr(div_up(nx, 32), div_up(ny, 8), B);
        if (s < s0_) {
            const int cx = nx_[s + 1], cy = ny_[s + 1];
            const dim3 zg(div_up(nx, 64), div_up(ny, 8), B);
            k_zoom_flow<<<zg, blk, 0, st>>>(U0, U1, N0, cx, cy, Uz, nx, ny, (float)nx / cx,
                                            (float)ny / cy, inv, ctrl);
            launches_ += 1;
        }
        k_cubic_pack<<<gr, blk, 0, st>>>(pyr + pyr_off_[s], lp, nx, ny, wc, N0);
        launches_ += 1;
        IterArgs ia{WR, U0, U1, P0, P1, N0, nx, ny, l_t, prm_.theta, taut, eps2, ctrl, part,
                    max_blocks_, iters, iter_stride_, 0};
        dim3 ig(div_up(nx, kIterTW), div_up(ny, kIterTH), B);
        const int cfg = tb_cfg_[s];
        const dim3 wb(kWarpTW, kWarpTH), wg(div_up(nx, kWarpTW), div_up(ny, kWarpTH), B);
        for (int wi = 0; wi < sw_[s]; wi++) {
            const int mode = wi > 0 ? kWarpFromU
                                    : (s == s0_ ? (warm_ ? kWarpFromUz : kWarpZero) : kWarpFromUz);
            mark_begin(-1);
            k_warp<<<wg, wb, 0, st>>>(pyr + pyr_off_[s], lp, wc, WR, U0, U1, Uz, P0, P1,
                                       N0, nx, ny, mode, wi == 0, ctrl, queue, left);
            mark_end();
            launches_ += 1;
            ia.stage = s * prm_.warps + wi;
            if (!trace_) {
                TbArgs ta{WR, U0, U1, P0, P1, N0, nx, ny, si_[s], l_t,
                          prm_.theta, taut, eps2, ctrl, part, max_blocks_ / kTbK, iters,
                          iter_stride_, ia.stage};
                tb_maps(ta, cfg, nx, ny, B, N0, P0, U0, WR, err_.device());
                const dim3 tg = tb_grid(cfg, nx, ny, B);
                mark_begin(s);
                if (cfg == kLevelCfg || cfg == kClusterCfg || queue_) {
                    // the whole stage in one launch
                    if (cfg == kLevelCfg || cfg == kClusterCfg)
                        tb_launch_cfg(cfg, tg, st, ta);
                    else
                        tb_launch_queue(cfg, tg, st, ta, queue, left, predict_, share_);
                    launches_ += 1;
                } else {
                    // blocked schedule: ceil(max/K) launches plus one for a
                    // possible re-run after a mid-block stop
                    const int nl = si_[s] > 0 ? div_up(si_[s], kTbK) + 1 : 0;
                    for (int it = 0; it < nl; it++) {
                        tb_launch_cfg(cfg, tg, st, ta);
                        launches_ += 1;
                    }
                }
                mark_end();
                continue;
            }
            for (int it = 0; it < prm_.max_iterations; it++) {
                mark_begin(s);
                k_tvl1_iter<kIterTW, kIterTH, kIterNT><<<ig, kIterNT, 0, st>>>(ia);
                mark_end();
                launches_ += 1;
                const int slot = (s * prm_.warps + wi) * prm_.max_iterations + it;
                k_energy<<<dim3(imin(energy_blocks_, div_up(nx * ny, kEnNT * 4)), B), kEnNT, 0,
                           st>>>(WR, U0, U1, N0, nx, ny, prm_.lambda, ctrl, part, max_blocks_,
                                 energy, energy_slots_, slot, it + 1);
                launches_ += 1;
            }
        }
    }
    // final energy at the finest scale, last warp: in the schedule of a traced
    // plan; otherwise on demand (compute_energy), when statistics are read
    if (trace_) {
        k_energy<<<dim3(energy_blocks_, B), kEnNT, 0, st>>>(WR, U0, U1, N0, w_, h_, prm_.lambda,
                                                            ctrl, part, max_blocks_, energy,
                                                            energy_slots_, -1, -1);
        launches_ += 1;
    }
    k_split<<<dim3(div_up(w_, 32), div_up(h_, 8), B), dim3(32, 8), 0, st>>>(
        U0, U1, N0, w_, h_, ar_.at<OutRef>(o_otab_), ctrl);
    launches_ += 1;
    OF_CUDA(cudaGetLastError());
}

// The schedule replayed as a CUDA graph with event nodes around every warp and
// inner-iteration launch (timings on the GPU timeline, no host gaps); returns
// per-kind totals (ms) and launch counts.
void TvPlan::profile(cudaStream_t st, oflow_tvl1_profile *out) {
    Prof p;
    cudaEvent_t t0, t1;
    OF_CUDA(cudaEventCreate(&t0));
    OF_CUDA(cudaEventCreate(&t1));
    auto cleanup = [&]() {
        prof_ = nullptr;
        for (auto &e : p.ev) cudaEventDestroy(e);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
    };
    try {
        Graph g;
        prof_ = &p;
        g.capture(st, [&](cudaStream_t s) {
            OF_CUDA(cudaEventRecordWithFlags(t0, s, cudaEventRecordExternal));
            record(s);
            OF_CUDA(cudaEventRecordWithFlags(t1, s, cudaEventRecordExternal));
        });
        prof_ = nullptr;
        upload_frames(st);
        g.launch(st);
        OF_CUDA(cudaStreamSynchronize(st));
        std::memset(out, 0, sizeof(*out));
        float ms = 0.0f;
        OF_CUDA(cudaEventElapsedTime(&ms, t0, t1));
        out->total_ms = ms;
        for (size_t k = 0; k < p.tag.size(); k++) {
            OF_CUDA(cudaEventElapsedTime(&ms, p.ev[2 * k], p.ev[2 * k + 1]));
            if (p.tag[k] < 0) {
                out->warp_ms += ms;
                out->warp_launches += 1;
            } else {
                out->iter_ms += ms;
                out->iter_ms_scale[p.tag[k]] += ms;
                out->iter_launches += 1;
            }
        }
        out->launches = launches_;
    } catch (...) {
        cleanup();
        throw;
    }
    cleanup();
}

// Re-arms every pair for a timing launch: iteration count 0, not stopped.
__global__ void k_ctrl_rearm(TvCtrl *ctrl, int B) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    ctrl[b].n = 0;
    ctrl[b].stop = 0;
    ctrl[b].redo = 0;
    ctrl[b].arrive = 0;
}

// Times every blocked-iteration configuration at every scale on the plan's
// current buffers (run a solve first so they hold real data) and keeps the
// fastest; best of `reps` single launches with all pairs active.
void TvPlan::autotune(cudaStream_t st, TuneTable *table, int reps) {
    const size_t N0 = N0_;
    TvCtrl *ctrl = ar_.at<TvCtrl>(o_ctrl_);
    cudaEvent_t e0, e1;
    OF_CUDA(cudaEventCreate(&e0));
    OF_CUDA(cudaEventCreate(&e1));
    const float l_t = prm_.lambda * prm_.theta, taut = prm_.tau / prm_.theta;
    const float eps2 = prm_.epsilon * prm_.epsilon;
    try {
        for (int s = 0; s < ns_; s++) {
            const int nx = nx_[s], ny = ny_[s];
            float best = 1e30f;
            int best_c = tb_cfg_[s];
            for (int c = 0; c < kNumIterCfgs; c++) {
                if (!cfg_valid(c, nx, ny)) continue;
                // per-iteration time: a tiled launch runs K iterations (no
                // stop); the whole-level kernel is given 2K
                const bool whole = c == kLevelCfg || c == kClusterCfg;
                const int iters_run = whole ? 2 * kTbK : kTbK;
                TbArgs ta{ar_.at<float4>(o_WR_), ubuf(0), ubuf(1), pbuf(0),
                          pbuf(1), N0,
                          nx, ny, whole ? iters_run : 1 << 30, l_t, prm_.theta, taut, -1.0f,
                          ctrl, ar_.at<double>(o_part_), max_blocks_ / kTbK, ar_.at<int>(o_iters_),
                          iter_stride_, 0};
                tb_maps(ta, c, nx, ny, B_, N0, pbuf(0), ubuf(0), ar_.at<float4>(o_WR_), err_.device());
                const dim3 tg = tb_grid(c, nx, ny, B_);
                float ms_min = 1e30f;
                for (int r = 0; r <= reps; r++) {  // first launch warms up
                    k_ctrl_rearm<<<div_up(B_, 128), 128, 0, st>>>(ctrl, B_);
                    OF_CUDA(cudaEventRecord(e0, st));
                    tb_launch_cfg(c, tg, st, ta);
                    OF_CUDA(cudaEventRecord(e1, st));
                    OF_CUDA(cudaEventSynchronize(e1));
                    float ms = 0.0f;
                    OF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                    if (r > 0) ms_min = ms < ms_min ? ms : ms_min;
                }
                ms_min /= (float)iters_run;
                if (ms_min < best) {
                    best = ms_min;
                    best_c = c;
                }
            }
            tb_cfg_[s] = best_c;
            if (table) (*table)[tune_key(nx, ny, B_)] = best_c;
        }
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    graph_.reset();  // the next run captures the new configurations
}

// Relative end-point difference of each pair's flow against another solve of
// the same pairs: sum ||(u, v) - (u', v')|| / sum ||(u', v')|| in double, one
// block per pair in a fixed order (the judge's decision is reproducible).
constexpr int kEpeNT = 1024;
__global__ void __launch_bounds__(kEpeNT) k_flow_rel_epe(const float *u, const float *v,
                                                         const float *pu, const float *pv,
                                                         size_t stride, int N, double *out) {
    __shared__ double sred[kEpeNT / 32];
    const size_t o = (size_t)blockIdx.x * stride;
    double d = 0.0, m = 0.0;
    for (int i = threadIdx.x; i < N; i += kEpeNT) {
        const double a = u[o + i], bb = v[o + i], pa = pu[o + i], pb = pv[o + i];
        d += sqrt((a - pa) * (a - pa) + (bb - pb) * (bb - pb));
        m += sqrt(pa * pa + pb * pb);
    }
    const double D = block_sum_double<kEpeNT>(d, sred);
    __syncthreads();
    const double M = block_sum_double<kEpeNT>(m, sred);
    if (threadIdx.x == 0) out[blockIdx.x] = M > 0.0 ? D / M : (D > 0.0 ? INFINITY : 0.0);
}

void TvPlan::rel_epe_against(const TvPlan &other, double *host_out, cudaStream_t st) {
    OF_CHECK(other.w_ == w_ && other.h_ == h_ && other.B_ == B_, "tvl1: plans of different shape");
    double *out = ar_.at<double>(o_tout_);
    k_flow_rel_epe<<<B_, kEpeNT, 0, st>>>(out_u(0), out_v(0), other.out_u(0), other.out_v(0), N0_,
                                          (int)N0_, out);
    OF_CUDA(cudaGetLastError());
    OF_CUDA(cudaMemcpyAsync(host_out, out, sizeof(double) * B_, cudaMemcpyDeviceToHost, st));
    OF_CUDA(cudaStreamSynchronize(st));
}

void TvPlan::true_energy(double *host_out, cudaStream_t st) {
    unsigned *arrive = ar_.at<unsigned>(o_tarr_);
    double *out = ar_.at<double>(o_tout_);
    OF_CUDA(cudaMemsetAsync(arrive, 0, sizeof(unsigned) * B_, st));
    k_energy_true<<<dim3(energy_blocks_, B_), kEnNT, 0, st>>>(
        ar_.at<float>(o_pyr_) + pyr_off_[0], N0_, ubuf(0), ubuf(1), N0_,
        w_, h_, prm_.lambda, ar_.at<TvCtrl>(o_ctrl_), ar_.at<double>(o_part_), max_blocks_,
        arrive, out);
    OF_CUDA(cudaGetLastError());
    OF_CUDA(cudaMemcpyAsync(host_out, out, sizeof(double) * B_, cudaMemcpyDeviceToHost, st));
    OF_CUDA(cudaStreamSynchronize(st));
}

void TvPlan::set_schedule(const int *warps, const int *iters) {
    OF_CHECK(!trace_, "tvl1: a traced plan runs the uniform schedule");
    for (int s = 0; s <= s0_; s++) {  // the scales this plan solves
        const int w = warps ? warps[s] : prm_.warps, n = iters ? iters[s] : prm_.max_iterations;
        OF_CHECK(w >= 1 && w <= prm_.warps, "tvl1: warps of a scale must be in [1, params.warps]");
        OF_CHECK(n >= 0, "tvl1: iterations of a scale < 0");
        if (w != sw_[s] || n != si_[s]) graph_.reset();
        sw_[s] = w;
        si_[s] = n;
    }
}

bool TvPlan::same_schedule(const int *warps, const int *iters) const {
    for (int s = 0; s <= s0_; s++) {
        if (sw_[s] != (warps ? warps[s] : prm_.warps)) return false;
        if (si_[s] != (iters ? iters[s] : prm_.max_iterations)) return false;
    }
    return true;
}

void TvPlan::run(cudaStream_t st) {
    upload_frames(st);
    if (!graph_.ready()) {
        graph_.capture(st, [&](cudaStream_t s) { record(s); });
        graph_launches_ = launches_;
    }
    graph_.launch(st);
    // Failure injection on the host: OFLOW_INJECT_TIMEOUT=1 raises the
    // plan's error flag as a kernel whose bounded wait gave up would, so the
    // report (OFLOW_ERR_TIMEOUT) and the recovery of the next call can be
    // tested without making any GPU wait run out.
    if (const char *e = getenv("OFLOW_INJECT_TIMEOUT"))
        if (atoi(e) == 1) err_.raise();
}

void TvPlan::compute_energy(cudaStream_t st) {
    if (trace_) return;  // the traced schedule computes it
    k_energy<<<dim3(energy_blocks_, B_), kEnNT, 0, st>>>(
        ar_.at<float4>(o_WR_), ubuf(0), ubuf(1), N0_, w_, h_, prm_.lambda, ar_.at<TvCtrl>(o_ctrl_),
        ar_.at<double>(o_part_), max_blocks_, ar_.at<double>(o_energy_), energy_slots_, 0, -1);
    OF_CUDA(cudaGetLastError());
}

void TvPlan::read_stats(int b, oflow_tvl1_stats *out, cudaStream_t st) const {
    std::vector<int> it(iter_stride_);
    OF_CUDA(cudaMemcpyAsync(it.data(), iters_dev() + (size_t)b * iter_stride_,
                            sizeof(int) * iter_stride_, cudaMemcpyDeviceToHost, st));
    TvCtrl c;
    OF_CUDA(cudaMemcpyAsync(&c, ar_.at<TvCtrl>(o_ctrl_) + b, sizeof(TvCtrl), cudaMemcpyDeviceToHost, st));
    OF_CUDA(cudaStreamSynchronize(st));
    std::memset(out, 0, sizeof(*out));
    out->nscales = ns_;
    out->warps = prm_.warps;
    for (int i = 0; i < iter_stride_; i++) out->iterations[i] = it[i];
    out->energy = c.energy;
}

void TvPlan::read_energy_trace(int b, double *dst, cudaStream_t st) const {
    OF_CHECK(trace_, "tvl1: plan was built without the energy trace");
    OF_CUDA(cudaMemcpyAsync(dst, ar_.at<double>(o_energy_) + (size_t)b * energy_slots_,
                            sizeof(double) * energy_slots_, cudaMemcpyDeviceToHost, st));
    OF_CUDA(cudaStreamSynchronize(st));
}

}  // namespace oflow
