// Shared device/host helpers for the optical-flow kernels (sm_100a).
//
// Arithmetic contract: every translation unit that includes this header is
// compiled with -fmad=false (no fused multiply-add) and IEEE division and
// square root, so each expression rounds exactly as the reference's x86
// build does.  Where the reference mixes double-precision literals into single
// precision code, the device code does the same in double.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "exact_math.cuh"

#include <climits>
#include <cmath>
#include <cstddef>
#include <cstring>

namespace oflow {

constexpr int kNumSMs = 148;


__host__ __device__ inline int div_up(int a, int b) { return (a + b - 1) / b; }
__host__ __device__ inline int imin(int a, int b) { return a < b ? a : b; }
__host__ __device__ inline int imax(int a, int b) { return a > b ? a : b; }

// float -> int toward zero, saturated so +-2 cannot overflow.  Out-of-range
// and NaN coordinates always end in the clamped (border) case, which is the
// result the reference gets on x86 as well.
__device__ __forceinline__ int trunc_sat(float f) {
    if (!(f == f)) return INT_MIN + 2;
    if (f >= 2147483520.0f) return INT_MAX - 2;
    if (f <= -2147483520.0f) return INT_MIN + 2;
    return (int)f;
}

__device__ __forceinline__ int clamp_flag(int x, int n, bool &out) {
    if (x < 0) { out = true; return 0; }
    if (x >= n) { out = true; return n - 1; }
    return x;
}

// Visits the inclusive rectangle [x0,x1] x [y0,y1] of a region of width RW
// with NT threads, one pixel per step (one division per call).
template <int NT, typename F>
__device__ __forceinline__ void for_rect(int x0, int x1, int y0, int y1, F &&f) {
    const int w = x1 - x0 + 1, n = w * (y1 - y0 + 1);
    if (n <= 0) return;
    const int t = threadIdx.x;
    int rx = x0 + t % w, ry = y0 + t / w;
    const int sx = NT % w, sy = NT / w;
    for (int k = t; k < n; k += NT) {
        f(rx, ry);
        rx += sx;
        ry += sy;
        if (rx > x1) {
            rx -= w;
            ry += 1;
        }
    }
}

// Keys cubic (a = -1/2) through v0..v3 at offset x from v1, with single
// precision differences and double precision for the rest, as in
// src/tvl1/sequential/bicubic_interpolation/bicubic_interpolation.cpp:38-46.
// The cell splits into the part that depends on the four samples only
// (cubic_coef: the cubic and quadratic coefficients in double, the single
// precision difference v2 - v0, and v1) and the evaluation at x
// (cubic_eval); cubic_cell is the two in sequence, with the operations and
// roundings of the reference's one expression.
struct CubicCoef {
    double c3, c2;
    float d20, v1;
};

__device__ __forceinline__ CubicCoef cubic_coef(float v0, float v1, float v2, float v3) {
    const float d20 = v2 - v0;
    const float d12 = v1 - v2;
    double c3 = 3.0 * (double)d12;
    c3 = c3 + (double)v3;
    c3 = c3 - (double)v0;
    double c2 = 2.0 * (double)v0;
    c2 = c2 - 5.0 * (double)v1;
    c2 = c2 + 4.0 * (double)v2;
    c2 = c2 - (double)v3;
    return CubicCoef{c3, c2, d20, v1};
}

// xd = (double)x, hx = 0.5 * xd (exact), shared by the cells of one sample.
__device__ __forceinline__ float cubic_eval(double c3, double c2, float d20, float v1, double xd,
                                            double hx) {
    c2 = c2 + xd * c3;
    const double t = (double)d20 + xd * c2;
    const double r = (double)v1 + hx * t;
    return (float)r;
}

__device__ __forceinline__ float cubic_cell(float v0, float v1, float v2, float v3, float x) {
    const double xd = x;
    const CubicCoef k = cubic_coef(v0, v1, v2, v3);
    return cubic_eval(k.c3, k.c2, k.d20, k.v1, xd, 0.5 * xd);
}

// Stencil of the reference's bicubic sample (bicubic_interpolation.cpp:74-128):
// columns/rows step away from zero by the coordinate's sign; the row above
// steps by the x sign (the reference's sx/sy mix-up, :92).  Returns false when
// border_out and any index was clamped (the sample is then 0).
struct BicubicStencil {
    int col[4];
    int row[4];
    float tx, ty;
};

__device__ __forceinline__ bool bicubic_stencil(float uu, float vv, int nx, int ny,
                                                bool border_out, BicubicStencil &s) {
    const int sx = (uu < 0) ? -1 : 1;
    const int sy = (vv < 0) ? -1 : 1;
    const int xi = trunc_sat(uu), yi = trunc_sat(vv);
    bool out = false;
    const int x = clamp_flag(xi, nx, out);
    const int y = clamp_flag(yi, ny, out);
    const int mx = clamp_flag(xi - sx, nx, out);
    const int my = clamp_flag(yi - sx, ny, out);
    const int dx = clamp_flag(xi + sx, nx, out);
    const int dy = clamp_flag(yi + sy, ny, out);
    const int ddx = clamp_flag(xi + 2 * sx, nx, out);
    const int ddy = clamp_flag(yi + 2 * sy, ny, out);
    if (out && border_out) return false;
    s.col[0] = mx; s.col[1] = x; s.col[2] = dx; s.col[3] = ddx;
    s.row[0] = my; s.row[1] = y; s.row[2] = dy; s.row[3] = ddy;
    s.tx = uu - (float)x;
    s.ty = vv - (float)y;
    return true;
}

// Scalar bicubic sample of a single-channel plane.
__device__ __forceinline__ float bicubic_at(const float *__restrict__ in, float uu, float vv,
                                            int nx, int ny, bool border_out) {
    BicubicStencil s;
    if (!bicubic_stencil(uu, vv, nx, ny, border_out, s)) return 0.0f;
    float v[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const float *col = in + s.col[c];
        v[c] = cubic_cell(__ldg(col + (size_t)nx * s.row[0]), __ldg(col + (size_t)nx * s.row[1]),
                          __ldg(col + (size_t)nx * s.row[2]), __ldg(col + (size_t)nx * s.row[3]),
                          s.ty);
    }
    return cubic_cell(v[0], v[1], v[2], v[3], s.tx);
}

// Bilinear sample, clamp-to-edge taps, coordinate first limited to [-1, n].
__device__ __forceinline__ float bilinear_clamped(const float *__restrict__ src, int w, int h,
                                                  float xf, float yf) {
    xf = fminf(fmaxf(xf, -1.0f), (float)w);
    yf = fminf(fmaxf(yf, -1.0f), (float)h);
    const float x0f = floorf(xf), y0f = floorf(yf);
    const float fx = xf - x0f, fy = yf - y0f;
    const int x0 = (int)x0f, y0 = (int)y0f;
    const int xa = imin(imax(x0, 0), w - 1), xb = imin(imax(x0 + 1, 0), w - 1);
    const int ya = imin(imax(y0, 0), h - 1), yb = imin(imax(y0 + 1, 0), h - 1);
    const float v00 = __ldg(src + (size_t)ya * w + xa), v10 = __ldg(src + (size_t)ya * w + xb);
    const float v01 = __ldg(src + (size_t)yb * w + xa), v11 = __ldg(src + (size_t)yb * w + xb);
    const float gx = 1.0f - fx, gy = 1.0f - fy;
    const float top = gx * v00 + fx * v10;
    const float bot = gx * v01 + fx * v11;
    return gy * top + fy * bot;
}

// Deterministic block reduction of one double per thread (fixed shuffle tree
// then a fixed pass over warps).  Result valid in thread 0.  `scratch` holds
// one double per warp.
template <int THREADS>
__device__ __forceinline__ double block_sum_double(double v, double *scratch) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < THREADS / 32; i++) r += scratch[i];
    }
    return r;
}

}  // namespace oflow
