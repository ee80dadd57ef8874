// Lucas-Kanade on B200: the reference's single-step solver over a frame ring
// (src/lk/cuda/lucaskanade.cu:54-71, kernels/kernels.cu:14-181) as one fused
// kernel, and a pyramidal, iterated variant built from the same steps.  The
// arithmetic contract is in common.cuh.
//
// The five window sums are accumulated per pixel in the reference's order
// (window rows, then columns), read from shared memory; a prefix-sum or
// separable box filter would change the rounding of det(A) and with it the
// flow wherever the structure tensor is near singular.
#include "common.cuh"
#include "hs.hpp"
#include "internal.hpp"
#include "lk.hpp"
#include "tvl1.hpp"

namespace oflow {

constexpr int kLTW = 32, kLTH = 8, kLNT = kLTW * kLTH;
constexpr int kLMaxC = 4, kLMaxF = 4, kLMaxT = 9;

struct LkTaps {
    float fs[9];
    float ft[9];
    int ns, nt;
};

int lk_taps(int spac, int temp, float *fs, float *ft) {
    static const float s1[] = {1.0f};
    static const float s3[] = {-1.0f / 2.0f, 0.0f, 1.0f / 2.0f};
    static const float s5[] = {1.0f / 12.0f, -2.0f / 3.0f, 0.0f, 2.0f / 3.0f, -1.0f / 12.0f};
    static const float s7[] = {-1.0f / 60.0f, 3.0f / 20.0f, -3.0f / 4.0f, 0.0f,
                               3.0f / 4.0f,   -3.0f / 20.0f, 1.0f / 60.0f};
    static const float s9[] = {1.0f / 280.0f, -4.0f / 105.0f, 1.0f / 5.0f, -4.0f / 5.0f, 0.0f,
                               4.0f / 5.0f,   -1.0f / 5.0f,   4.0f / 105.0f, -1.0f / 280.0f};
    static const float t2[] = {-1.0f, 1.0f};
    // central-difference tables of src/lk/cuda/lucaskanade.cu:79-161
    const float *S = spac == 1 ? s1 : spac == 3 ? s3 : spac == 5 ? s5 : spac == 7 ? s7
                                                                                    : spac == 9 ? s9 : nullptr;
    const float *T = temp == 1 ? s1 : temp == 2 ? t2 : temp == 3 ? s3 : temp == 5 ? s5
                                                                                   : temp == 7 ? s7
                                                                                               : temp == 9 ? s9
                                                                                                           : nullptr;
    if (!S || !T) return -1;
    for (int i = 0; i < spac; i++) fs[i] = S[i];
    for (int i = 0; i < temp; i++) ft[i] = T[i];
    return 0;
}

// Window sums in the reference order and the closed-form 2x2 solve
// (kernels.cu:150-179).  gx/gy/gt: region planes of width RW.
__device__ __forceinline__ void lk_window_solve(const float *gx, const float *gy, const float *gt,
                                                int RW, int cidx, int c, float &vx, float &vy) {
    float sxx = 0.0f, sxy = 0.0f, syy = 0.0f, sxt = 0.0f, syt = 0.0f;
    for (int ii = -c; ii <= c; ii++) {
        const int row = cidx + ii * RW;
        for (int jj = -c; jj <= c; jj++) {
            const int q = row + jj;
            const float ix = gx[q], iy = gy[q], it = gt[q];
            sxx += ix * ix;
            sxy += ix * iy;
            syy += iy * iy;
            sxt += ix * it;
            syt += iy * it;
        }
    }
    const float det = (sxx * syy - sxy * sxy);
    vx = 0.0f;
    vy = 0.0f;
    if (det != 0.0f) {
        vx = 1.0f / det * (syy * (-sxt) + (-sxy) * (-syt));
        vy = 1.0f / det * ((-sxy) * (-sxt) + sxx * (-syt));
    }
}

// Single step over a ring of T uint8 frames (slot k at ring + k*N); the newest
// frame is in slot iframe % T.  One kernel: spatial FIR of the oldest frame,
// temporal FIR over the ring, window sums and solve.  Pixels closer than the
// window radius to the border get 0.
__global__ void __launch_bounds__(kLNT) k_lk_step(const uint8_t *__restrict__ ring, int T,
                                                  int iframe, int nx, int ny, const __grid_constant__ LkTaps taps,
                                                  int c, float *Vx, float *Vy) {
    constexpr int RWm = kLTW + 2 * kLMaxC, RHm = kLTH + 2 * kLMaxC;
    constexpr int FWm = RWm + 2 * kLMaxF, FHm = RHm + 2 * kLMaxF;
    __shared__ float sf[FWm * FHm];
    __shared__ float gx[RWm * RHm], gy[RWm * RHm], gt[RWm * RHm];
    const int fc = (taps.ns - 1) / 2;
    const int RW = kLTW + 2 * c, RH = kLTH + 2 * c;
    const int FW = RW + 2 * fc, FH = RH + 2 * fc;
    const size_t N = (size_t)nx * ny;
    const uint8_t *old = ring + (size_t)((iframe + 1) % T) * N;
    const int fx0 = blockIdx.x * kLTW - c - fc, fy0 = blockIdx.y * kLTH - c - fc;
    for (int i = threadIdx.x; i < FW * FH; i += kLNT) {
        const int x = fx0 + i % FW, y = fy0 + i / FW;
        sf[i] = (x >= 0 && x < nx && y >= 0 && y < ny) ? (float)old[(size_t)y * nx + x] : 0.0f;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < RW * RH; i += kLNT) {
        const int rx = i % RW, ry = i / RW;
        const int x = fx0 + fc + rx, y = fy0 + fc + ry;
        if (x < 0 || x >= nx || y < 0 || y >= ny) continue;
        const float *f = sf + (ry + fc) * FW + (rx + fc);
        float ax = 0.0f, ay = 0.0f;
        for (int k = 0; k < taps.ns; k++) {
            const int xx = x + k - fc, yy = y + k - fc;
            if (xx >= 0 && xx < nx) ax += f[k - fc] * taps.fs[k];
            if (yy >= 0 && yy < ny) ay += f[(k - fc) * FW] * taps.fs[k];
        }
        float at = 0.0f;
        for (int fr = 0; fr < T; fr++)
            at += taps.ft[fr] * (float)ring[(size_t)((fr + iframe + 1) % T) * N + (size_t)y * nx + x];
        gx[i] = ax;
        gy[i] = ay;
        gt[i] = at;
    }
    __syncthreads();
    const int x = blockIdx.x * kLTW + threadIdx.x % kLTW, y = blockIdx.y * kLTH + threadIdx.x / kLTW;
    if (x >= nx || y >= ny) return;
    float vx = 0.0f, vy = 0.0f;
    if (x >= c && y >= c && x < nx - c && y < ny - c)
        lk_window_solve(gx, gy, gt, RW, (threadIdx.x / kLTW + c) * RW + threadIdx.x % kLTW + c, c,
                        vx, vy);
    Vx[(size_t)y * nx + x] = vx;
    Vy[(size_t)y * nx + x] = vy;
}

// Spatial FIR (zero padding by dropped taps) of a float plane -> float2 (Ix, Iy),
// NS taps at compile time (every tap added, the zero one too, as the
// reference does); pixels at least NS/2 from every border skip the tests.
template <int NS>
__global__ void k_lk_grad(const float *__restrict__ src, size_t sstride, int nx, int ny,
                          const __grid_constant__ LkTaps taps, float2 *G, size_t gstride) {
    constexpr int FC = (NS - 1) / 2;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= nx || y >= ny) return;
    const float *f = src + (size_t)blockIdx.z * sstride;
    float ax = 0.0f, ay = 0.0f;
    if (x >= FC && x < nx - FC && y >= FC && y < ny - FC) {
        const float *row = f + (size_t)y * nx + x - FC, *col = f + (size_t)(y - FC) * nx + x;
#pragma unroll
        for (int k = 0; k < NS; k++) {
            ax += __ldg(row + k) * taps.fs[k];
            ay += __ldg(col + (size_t)k * nx) * taps.fs[k];
        }
    } else {
#pragma unroll
        for (int k = 0; k < NS; k++) {
            const int xx = x + k - FC, yy = y + k - FC;
            if (xx >= 0 && xx < nx) ax += __ldg(f + (size_t)y * nx + xx) * taps.fs[k];
            if (yy >= 0 && yy < ny) ay += __ldg(f + (size_t)yy * nx + x) * taps.fs[k];
        }
    }
    G[(size_t)blockIdx.z * gstride + (size_t)y * nx + x] = make_float2(ax, ay);
}

static void launch_lk_grad(dim3 g, dim3 blk, cudaStream_t st, const float *src, size_t sstride,
                           int nx, int ny, const LkTaps &taps, float2 *G, size_t gstride) {
    switch (taps.ns) {
        case 1: k_lk_grad<1><<<g, blk, 0, st>>>(src, sstride, nx, ny, taps, G, gstride); break;
        case 3: k_lk_grad<3><<<g, blk, 0, st>>>(src, sstride, nx, ny, taps, G, gstride); break;
        case 5: k_lk_grad<5><<<g, blk, 0, st>>>(src, sstride, nx, ny, taps, G, gstride); break;
        case 7: k_lk_grad<7><<<g, blk, 0, st>>>(src, sstride, nx, ny, taps, G, gstride); break;
        default: k_lk_grad<9><<<g, blk, 0, st>>>(src, sstride, nx, ny, taps, G, gstride); break;
    }
}

// Window sums and the 2x2 solve of P vertically adjacent pixels (column cidx,
// rows of centres crow .. crow+P-1 in shared memory): each window element is
// loaded and its five products formed once for every pixel whose window holds
// it; each pixel still adds them in the reference's row-major order
// (kernels.cu:150-179), so its sums are those of lk_window_solve.
template <int C, int P>
__device__ __forceinline__ void lk_window_solve_p(const float *gx, const float *gy, const float *gt,
                                                  int RW, int top, float (&vx)[P], float (&vy)[P]) {
    float sxx[P], sxy[P], syy[P], sxt[P], syt[P];
#pragma unroll
    for (int k = 0; k < P; k++) sxx[k] = sxy[k] = syy[k] = sxt[k] = syt[k] = 0.0f;
#pragma unroll
    for (int r = 0; r < 2 * C + P; r++) {
        const int row = top + r * RW;
#pragma unroll
        for (int jj = 0; jj <= 2 * C; jj++) {
            const float ix = gx[row + jj], iy = gy[row + jj], it = gt[row + jj];
            const float pxx = ix * ix, pxy = ix * iy, pyy = iy * iy, pxt = ix * it, pyt = iy * it;
#pragma unroll
            for (int k = 0; k < P; k++)
                if (r - k >= 0 && r - k <= 2 * C) {
                    sxx[k] += pxx;
                    sxy[k] += pxy;
                    syy[k] += pyy;
                    sxt[k] += pxt;
                    syt[k] += pyt;
                }
        }
    }
#pragma unroll
    for (int k = 0; k < P; k++) {
        const float det = (sxx[k] * syy[k] - sxy[k] * sxy[k]);
        vx[k] = 0.0f;
        vy[k] = 0.0f;
        if (det != 0.0f) {
            vx[k] = 1.0f / det * (syy[k] * (-sxt[k]) + (-sxy[k]) * (-syt[k]));
            vy[k] = 1.0f / det * ((-sxy[k]) * (-sxt[k]) + sxx[k] * (-syt[k]));
        }
    }
}

// One refinement of pyramidal LK: warp I1 by the current flow (bilinear,
// clamp-to-edge), It = 0 + (-1)*I0 + 1*I1w, window solve, Uout = Uin + d.
// Tile 32 x kPTH with the window radius C as halo; a thread solves PP
// vertically adjacent pixels (lk_window_solve_p): 4 when a launch has tiles
// enough to fill the GPU (the elements of eight window rows loaded and
// multiplied once for four pixels: 29.0k against 28.0k pairs/s on 64 pairs of
// 640x480), else 2 (twice the threads: 9.7k against 9.2k pairs/s for one
// pair).  (Window sums read from precomputed product planes measured slower:
// 18.2k against 21.4k pairs/s batched; five loads per window element instead
// of three bound the LSU pipe.)
constexpr int kPTW = 32, kPTH = 32;
template <int C, int PP>
__global__ void __launch_bounds__(kPTW * kPTH / PP) k_pyrlk_iter(const float *__restrict__ pyr, size_t lp,
                                                                 const float2 *__restrict__ G, size_t gstride,
                                                                 const float2 *__restrict__ Uin,
                                                                 float2 *Uout, size_t ustride, int nx,
                                                                 int ny) {
    constexpr int kPNT = kPTW * kPTH / PP;
    constexpr int RW = kPTW + 2 * C, RH = kPTH + 2 * C;
    __shared__ float gx[RW * RH], gy[RW * RH], gt[RW * RH];
    const int b = blockIdx.z;
    const float *I0 = pyr + (size_t)(2 * b) * lp;
    const float *I1 = pyr + (size_t)(2 * b + 1) * lp;
    const float2 *Gb = G + (size_t)b * gstride;
    const float2 *Ub = Uin + (size_t)b * ustride;
    const int x0 = blockIdx.x * kPTW - C, y0 = blockIdx.y * kPTH - C;
    for (int i = threadIdx.x; i < RW * RH; i += kPNT) {
        const int x = x0 + i % RW, y = y0 + i / RW;
        if (x < 0 || x >= nx || y < 0 || y >= ny) {
            // read only by the sums of border pixels, whose results are not used
            gx[i] = gy[i] = gt[i] = 0.0f;
            continue;
        }
        const size_t p = (size_t)y * nx + x;
        const float2 u = Ub[p];
        const float w = bilinear_clamped(I1, nx, ny, (float)x + u.x, (float)y + u.y);
        float it = 0.0f;
        it += -1.0f * __ldg(I0 + p);
        it += 1.0f * w;
        const float2 g = Gb[p];
        gx[i] = g.x;
        gy[i] = g.y;
        gt[i] = it;
    }
    __syncthreads();
    const int tx = threadIdx.x % kPTW, ty = (threadIdx.x / kPTW) * PP;
    const int x = blockIdx.x * kPTW + tx, yb = blockIdx.y * kPTH + ty;
    if (x >= nx || yb >= ny) return;
    float dx[PP], dy[PP];
    // top-left of the first pixel's window: row ty, column tx of the region
    lk_window_solve_p<C, PP>(gx, gy, gt, RW, ty * RW + tx, dx, dy);
#pragma unroll
    for (int k = 0; k < PP; k++) {
        const int y = yb + k;
        if (y >= ny) break;
        const bool in = x >= C && y >= C && x < nx - C && y < ny - C;
        const size_t q = (size_t)y * nx + x;
        const float2 u = Ub[q];
        Uout[(size_t)b * ustride + q] = make_float2(u.x + (in ? dx[k] : 0.0f), u.y + (in ? dy[k] : 0.0f));
    }
}

static void launch_pyrlk_iter(int c, dim3 g, cudaStream_t st, const float *pyr, size_t lp,
                              const float2 *G, size_t gstride, const float2 *Uin, float2 *Uout,
                              size_t ustride, int nx, int ny) {
    const bool wide = (size_t)g.x * g.y * g.z > 4 * (size_t)kNumSMs;
#define OF_PYRLK(C)                                                                                  \
    if (wide)                                                                                        \
        k_pyrlk_iter<C, 4><<<g, kPTW * kPTH / 4, 0, st>>>(pyr, lp, G, gstride, Uin, Uout, ustride, nx, ny); \
    else                                                                                             \
        k_pyrlk_iter<C, 2><<<g, kPTW * kPTH / 2, 0, st>>>(pyr, lp, G, gstride, Uin, Uout, ustride, nx, ny);
    switch (c) {
        case 0: OF_PYRLK(0) break;
        case 1: OF_PYRLK(1) break;
        case 2: OF_PYRLK(2) break;
        case 3: OF_PYRLK(3) break;
        default: OF_PYRLK(4) break;
    }
#undef OF_PYRLK
}

// ================================================================ host plans
static LkTaps make_lk_taps(int spac, int temp) {
    LkTaps t{};
    if (lk_taps(spac, temp, t.fs, t.ft) != 0) throw Error(OFLOW_ERR_BAD_ARG, "lk: filter size not supported");
    t.ns = spac;
    t.nt = temp;
    return t;
}

LkPlan::LkPlan(int w, int h, const oflow_lk_params &prm) : w_(w), h_(h), prm_(prm) {
    OF_CHECK(prm.window >= 1 && (prm.window & 1) && (prm.window - 1) / 2 <= kLMaxC,
             "lk: window must be odd and at most 9");
    OF_CHECK(prm.temp >= 1 && prm.temp <= kLMaxT, "lk: temporal filter size out of range");
    make_lk_taps(prm.spac, prm.temp);
    OF_CHECK(w >= prm.window && h >= prm.window && w >= prm.spac && h >= prm.spac,
             "lk: frame smaller than the window or filter");
    N_ = (size_t)w * h;
    o_ring_ = ar_.reserve((size_t)prm.temp * N_);
    o_out_ = ar_.reserve(2 * N_ * 4);
    ar_.commit();
}

uint8_t *LkPlan::ring_slot(int k) const { return ar_.at<uint8_t>(o_ring_) + (size_t)k * N_; }
const float *LkPlan::out_u() const { return ar_.at<float>(o_out_); }
const float *LkPlan::out_v() const { return ar_.at<float>(o_out_) + N_; }

void LkPlan::run(int iframe, cudaStream_t st) {
    const LkTaps taps = make_lk_taps(prm_.spac, prm_.temp);
    dim3 g(div_up(w_, kLTW), div_up(h_, kLTH));
    float *o = ar_.at<float>(o_out_);
    k_lk_step<<<g, kLNT, 0, st>>>(ar_.at<uint8_t>(o_ring_), prm_.temp, iframe, w_, h_, taps,
                                  (prm_.window - 1) / 2, o, o + N_);
    OF_CUDA(cudaGetLastError());
}

PyrLkPlan::PyrLkPlan(int w, int h, int B, int dtype, const oflow_lk_params &prm)
    : w_(w), h_(h), B_(B), dtype_(dtype), prm_(prm) {
    OF_CHECK(B >= 1, "pyrlk: empty batch");
    OF_CHECK(prm.window >= 1 && (prm.window & 1) && (prm.window - 1) / 2 <= kLMaxC,
             "pyrlk: window must be odd and at most 9");
    OF_CHECK(prm.levels >= 1 && prm.levels <= 16, "pyrlk: levels out of range");
    OF_CHECK(prm.iters >= 0, "pyrlk: iters < 0");
    make_lk_taps(prm.spac, 2);
    taps_ = make_zoom_taps(0.5f);
    L_ = prm.levels;
    W_[0] = w;
    H_[0] = h;
    for (int l = 1; l < L_; l++) tvl1_zoom_size(W_[l - 1], H_[l - 1], &W_[l], &H_[l], 0.5f);
    for (int l = 0; l + 1 < L_; l++)
        OF_CHECK(taps_.size <= W_[l] && taps_.size <= H_[l], "pyrlk: level smaller than the Gaussian window");
    for (int l = 0; l < L_; l++)
        OF_CHECK(W_[l] >= prm.window && H_[l] >= prm.window, "pyrlk: level smaller than the window");
    N_ = (size_t)w * h;
    size_t acc = 0;
    for (int l = 0; l < L_; l++) {
        pyr_off_[l] = acc;
        acc += (size_t)2 * B * W_[l] * H_[l];
    }
    const size_t esz = dtype == OFLOW_U8 ? 1 : 4;
    o_raw_ = ar_.reserve(2 * B * N_ * esz);
    o_T_ = ar_.reserve(2 * B * N_ * 4);
    o_pyr_ = ar_.reserve(acc * 4);
    o_G_ = ar_.reserve(B * N_ * 8);
    o_U0_ = ar_.reserve(B * N_ * 8);
    o_U1_ = ar_.reserve(B * N_ * 8);
    o_out_ = ar_.reserve(2 * B * N_ * 4);
    o_ftab_ = ar_.reserve(sizeof(FrameRef) * 2 * B);
    o_otab_ = ar_.reserve(sizeof(OutRef) * B);
    ar_.commit();
    io_.init(ar_.at<FrameRef>(o_ftab_), ar_.at<OutRef>(o_otab_), B);
    for (int b = 0; b < B; b++) {
        bind_raw(b, 0);
        bind_raw(b, 1);
        bind_own_out(b);
    }
    // the default tables are valid for schedules recorded into a caller's graph
    io_.upload(nullptr);
    OF_CUDA(cudaStreamSynchronize(nullptr));
}

void PyrLkPlan::bind_frame(int b, int k, const void *p, int pitch) { io_.set_frame(b, k, p, pitch ? pitch : w_); }
void PyrLkPlan::bind_raw(int b, int k) { io_.set_frame(b, k, raw_input(b, k), w_); }
void PyrLkPlan::bind_out(int b, float *u, float *v, int pitch) { io_.set_out(b, u, v, pitch ? pitch : w_); }
void PyrLkPlan::bind_own_out(int b) {
    float *o = ar_.at<float>(o_out_);
    io_.set_out(b, o + (size_t)b * N_, o + (size_t)(B_ + b) * N_, w_);
}

void *PyrLkPlan::raw_input(int b, int k) const {
    const size_t esz = dtype_ == OFLOW_U8 ? 1 : 4;
    return ar_.at<char>(o_raw_) + (size_t)(2 * b + k) * N_ * esz;
}
const float *PyrLkPlan::out_u(int b) const { return ar_.at<float>(o_out_) + (size_t)b * N_; }
const float *PyrLkPlan::out_v(int b) const { return ar_.at<float>(o_out_) + (size_t)(B_ + b) * N_; }

void PyrLkPlan::record(cudaStream_t st) {
    const int B = B_;
    float *pyr = ar_.at<float>(o_pyr_);
    float *T = ar_.at<float>(o_T_);
    float2 *G = ar_.at<float2>(o_G_);
    float2 *U[2] = {ar_.at<float2>(o_U0_), ar_.at<float2>(o_U1_)};
    const LkTaps taps = make_lk_taps(prm_.spac, 2);
    // frames through the frame table (device frames in place, or staged)
    launch_ingest_tab(io_.frames(), dtype_, w_, h_, pyr, N_, 2 * B, st);
    for (int l = 1; l < L_; l++) {
        const size_t sp = (size_t)W_[l - 1] * H_[l - 1], dp = (size_t)W_[l] * H_[l];
        launch_zoom_out(pyr + pyr_off_[l - 1], sp, W_[l - 1], H_[l - 1], T, pyr + pyr_off_[l], dp,
                        W_[l], H_[l], 0.5f, taps_, 2 * B, st);
    }
    int cur = 0;
    OF_CUDA(cudaMemsetAsync(U[cur], 0, B * N_ * 8, st));
    const int c = (prm_.window - 1) / 2;
    for (int l = L_ - 1; l >= 0; l--) {
        const int lw = W_[l], lh = H_[l];
        const size_t lp = (size_t)lw * lh;
        dim3 blk(32, 8), g(div_up(lw, 32), div_up(lh, 8), B);
        // Ix, Iy of I0: plane 2b of the level, so a stride of two planes
        launch_lk_grad(g, blk, st, pyr + pyr_off_[l], 2 * lp, lw, lh, taps, G, N_);
        dim3 ig(div_up(lw, kPTW), div_up(lh, kPTH), B);
        for (int r = 0; r < prm_.iters; r++) {
            launch_pyrlk_iter(c, ig, st, pyr + pyr_off_[l], lp, G, N_, U[cur], U[cur ^ 1], N_, lw, lh);
            cur ^= 1;
        }
        if (l > 0) {
            const float sx = (float)W_[l - 1] / (float)lw;
            const float sy = (float)H_[l - 1] / (float)lh;
            launch_upscale2(U[cur], N_, lw, lh, U[cur ^ 1], N_, W_[l - 1], H_[l - 1], sx, sy, B, st);
            cur ^= 1;
        }
    }
    launch_split_tab(U[cur], N_, w_, h_, io_.outs(), B, st);
    OF_CUDA(cudaGetLastError());
}

void PyrLkPlan::run(cudaStream_t st) {
    io_.upload(st);
    if (!graph_.ready()) graph_.capture(st, [&](cudaStream_t s) { record(s); });
    graph_.launch(st);
}

}  // namespace oflow
