/*
 * CPU oracle for TV-L1, Horn-Schunck and Lucas-Kanade.  TEST INFRASTRUCTURE
 * ONLY (the checker): the product never links or calls it.  See oracle.h for
 * the contract.  Every function cites the reference lines it restates; paths are
 * relative to the reference project root.
 */
#include "oracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

static float *falloc(size_t n) { return (float *)calloc(n ? n : 1, sizeof(float)); }

static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }

/* ===================================================================== */
/* TV-L1                                                                  */
/* ===================================================================== */

/* Window of the separable Gaussian: (int)(5*sigma)+1 taps on each side,
 * counting the centre (src/tvl1/sequential/mask/mask.cpp:227, mask.hpp:7). */
int orc_gaussian_window(double sigma) { return (int)(5.0 * sigma) + 1; }

/* Normalised half-kernel in double (mask.cpp:225-244): B[i] = exp(-i^2/(2s^2))
 * / (s*sqrt(2pi)), divided by 2*sum(B) - B[0] (sum taken left to right, as the
 * BLAS dasum, then a dscal by the reciprocal). */
static int gauss_taps(double sigma, double *B) {
    const double den = 2 * sigma * sigma;
    const double spi = sigma * sqrt(M_PI * 2);
    const int size = orc_gaussian_window(sigma);
    for (int i = 0; i < size; i++) B[i] = 1 / spi * exp(-i * i / den);
    double norm = 0.0;
    for (int i = 0; i < size; i++) norm += fabs(B[i]);
    norm = norm * 2 - B[0];
    const double s = 1 / norm;
    for (int i = 0; i < size; i++) B[i] = s * B[i];
    return size;
}

/* Mirror used by the Gaussian's line buffer (mask.cpp:250-256, 271-277):
 * before the start it reflects without repeating the edge sample
 * (x = -k reads k); past the end it reflects with the edge sample repeated
 * (x = n + k reads n - 1 - k). */
static inline int gauss_mirror(int x, int n) {
    if (x < 0) return -x;
    if (x >= n) return 2 * n - 1 - x;
    return x;
}

/* One 1-D pass over `line` (n samples, stride 1) into `dst`. */
static void gauss_line(const float *line, float *dst, int n, const double *B, int size) {
    for (int x = 0; x < n; x++) {
        double sum = B[0] * line[x];
        for (int j = 1; j < size; j++) {
            const float pair = line[gauss_mirror(x - j, n)] + line[gauss_mirror(x + j, n)];
            sum += B[j] * pair;
        }
        dst[x] = (float)sum;
    }
}

/* In-place separable Gaussian, rows then columns (mask.cpp:204-274).  Returns
 * -1 where the reference would terminate or read outside the image (window
 * wider than the width, mask.cpp:231; or taller than the height). */
int orc_gaussian(float *I, int nx, int ny, double sigma) {
    double B[64];
    if (orc_gaussian_window(sigma) > 64) return -1;
    const int size = gauss_taps(sigma, B);
    if (size > nx || size > ny) return -1;
    const int m = nx > ny ? nx : ny;
    float *line = falloc((size_t)m), *out = falloc((size_t)m);
    for (int y = 0; y < ny; y++) {
        memcpy(line, I + (size_t)y * nx, sizeof(float) * nx);
        gauss_line(line, I + (size_t)y * nx, nx, B, size);
    }
    for (int x = 0; x < nx; x++) {
        for (int y = 0; y < ny; y++) line[y] = I[(size_t)y * nx + x];
        gauss_line(line, out, ny, B, size);
        for (int y = 0; y < ny; y++) I[(size_t)y * nx + x] = out[y];
    }
    free(line);
    free(out);
    return 0;
}

/* Keys cubic through v[0..3] at offset x in [0,1) from v[1], with the
 * reference's mix of single and double precision
 * (src/tvl1/sequential/bicubic_interpolation/bicubic_interpolation.cpp:38-46):
 * the differences v2-v0 and v1-v2 are single, everything else double. */
static float cubic_cell(const float v[4], float x) {
    const double xd = x;
    const float d20 = v[2] - v[0];
    const float d12 = v[1] - v[2];
    double c3 = 3.0 * d12;
    c3 = c3 + v[3];
    c3 = c3 - v[0];
    double c2 = 2.0 * v[0];
    c2 = c2 - 5.0 * v[1];
    c2 = c2 + 4.0 * v[2];
    c2 = c2 - v[3];
    c2 = c2 + xd * c3;
    const double t = d20 + xd * c2;
    const double r = v[1] + (0.5 * xd) * t;
    return (float)r;
}

/* float -> int truncation toward zero, saturated so that +/-2 stays in range
 * (out-of-range values only ever land in the clamped, zeroed case). */
static inline int trunc_sat(float f) {
    if (!(f == f)) return INT_MIN + 2;
    if (f >= 2147483520.0f) return INT_MAX - 2;
    if (f <= -2147483520.0f) return INT_MIN + 2;
    return (int)f;
}

/* Neumann clamp that records whether clamping happened (bicubic_interpolation
 * .cpp:17-30: `out` is sticky over all eight calls). */
static inline int clamp_flag(int x, int n, int *out) {
    if (x < 0) { *out = 1; return 0; }
    if (x >= n) { *out = 1; return n - 1; }
    return x;
}

/* bicubic_interpolation.cpp:74-128.  The stencil steps away from zero by the
 * sign of the coordinate; the row below `y` steps by sx, not sy (:92). */
float orc_bicubic_at(const float *in, float uu, float vv, int nx, int ny, int border_out) {
    const int sx = (uu < 0) ? -1 : 1;
    const int sy = (vv < 0) ? -1 : 1;
    const int xi = trunc_sat(uu), yi = trunc_sat(vv);
    int out = 0;
    const int x = clamp_flag(xi, nx, &out);
    const int y = clamp_flag(yi, ny, &out);
    const int mx = clamp_flag(xi - sx, nx, &out);
    const int my = clamp_flag(yi - sx, ny, &out);
    const int dx = clamp_flag(xi + sx, nx, &out);
    const int dy = clamp_flag(yi + sy, ny, &out);
    const int ddx = clamp_flag(xi + 2 * sx, nx, &out);
    const int ddy = clamp_flag(yi + 2 * sy, ny, &out);
    if (out && border_out) return 0.0f;
    const int cols[4] = {mx, x, dx, ddx};
    const int rows[4] = {my, y, dy, ddy};
    const float ty = vv - (float)y, tx = uu - (float)x;
    float col[4], v[4];
    for (int c = 0; c < 4; c++) {
        for (int r = 0; r < 4; r++) col[r] = in[cols[c] + (size_t)nx * rows[r]];
        v[c] = cubic_cell(col, ty);
    }
    return cubic_cell(v, tx);
}

/* bicubic_interpolation.cpp:141-163: sample `in` at (j+u, i+v). */
void orc_bicubic_warp(const float *in, const float *u, const float *v, float *out, int nx,
                      int ny, int border_out) {
    for (int i = 0; i < ny; i++)
        for (int j = 0; j < nx; j++) {
            const size_t p = (size_t)i * nx + j;
            const float uu = (float)j + u[p];
            const float vv = (float)i + v[p];
            out[p] = orc_bicubic_at(in, uu, vv, nx, ny, border_out);
        }
}

/* src/tvl1/sequential/zoom/zoom.hpp:14-26 */
void orc_zoom_size(int nx, int ny, int *nxx, int *nyy, float factor) {
    *nxx = (int)((float)nx * factor + 0.5);
    *nyy = (int)((float)ny * factor + 0.5);
}

/* zoom.cpp:20-53: Gaussian with sigma = 0.6*sqrt(1/f^2 - 1) (rounded to
 * single), then bicubic samples at (j/f, i/f) without border zeroing. */
int orc_zoom_out(const float *I, float *Iout, int nx, int ny, float factor) {
    int nxx, nyy;
    orc_zoom_size(nx, ny, &nxx, &nyy, factor);
    const float sigma = (float)(0.6f * sqrt(1.0 / (factor * factor) - 1.0));
    float *Is = falloc((size_t)nx * ny);
    memcpy(Is, I, sizeof(float) * (size_t)nx * ny);
    if (orc_gaussian(Is, nx, ny, sigma) != 0) { free(Is); return -1; }
    for (int i1 = 0; i1 < nyy; i1++)
        for (int j1 = 0; j1 < nxx; j1++) {
            const float i2 = (float)i1 / factor;
            const float j2 = (float)j1 / factor;
            Iout[(size_t)i1 * nxx + j1] = orc_bicubic_at(Is, j2, i2, nx, ny, 0);
        }
    free(Is);
    return 0;
}

/* zoom.cpp:61-85: bicubic samples at (j/fx, i/fy), fx = nxx/nx in single. */
void orc_zoom_in(const float *I, float *Iout, int nx, int ny, int nxx, int nyy) {
    const float fx = (float)nxx / nx;
    const float fy = (float)nyy / ny;
    for (int i1 = 0; i1 < nyy; i1++)
        for (int j1 = 0; j1 < nxx; j1++) {
            const float i2 = (float)i1 / fy;
            const float j2 = (float)j1 / fx;
            Iout[(size_t)i1 * nxx + j1] = orc_bicubic_at(I, j2, i2, nx, ny, 0);
        }
}

/* mask.cpp:139-196: 0.5*(f[+1]-f[-1]), one-sided at the borders.  The
 * one-sided forms are exactly the central form with clamped indices. */
void orc_centered_gradient(const float *in, float *dx, float *dy, int nx, int ny) {
    for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
            const size_t row = (size_t)y * nx;
            const float ddx = in[row + imin(x + 1, nx - 1)] - in[row + imax(x - 1, 0)];
            const float ddy = in[(size_t)imin(y + 1, ny - 1) * nx + x] -
                              in[(size_t)imax(y - 1, 0) * nx + x];
            dx[row + x] = (float)(0.5 * ddx);
            dy[row + x] = (float)(0.5 * ddy);
        }
}

/* Backward-difference divergence with the reference's border cases, each
 * evaluated in the same order as written there (mask.cpp:31-90). */
static inline float div_at(const float *v1, const float *v2, int x, int y, int nx, int ny) {
    const size_t p = (size_t)y * nx + x;
    const int left = x == 0, right = x == nx - 1, top = y == 0, bottom = y == ny - 1;
    if (!left && !right && !top && !bottom) return (v1[p] - v1[p - 1]) + (v2[p] - v2[p - nx]);
    if (top && !left && !right) return v1[p] - v1[p - 1] + v2[p];
    if (bottom && !left && !right) return v1[p] - v1[p - 1] - v2[p - nx];
    if (left && !top && !bottom) return v1[p] + v2[p] - v2[p - nx];
    if (right && !top && !bottom) return -v1[p - 1] + v2[p] - v2[p - nx];
    if (left && top) return v1[p] + v2[p];
    if (right && top) return -v1[p - 1] + v2[p];
    if (left && bottom) return v1[p] - v2[p - nx];
    return -v1[p - 1] - v2[p - nx];
}

void orc_divergence(const float *v1, const float *v2, float *div, int nx, int ny) {
    for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) div[(size_t)y * nx + x] = div_at(v1, v2, x, y, nx, ny);
}

/* mask.cpp:86-144: forward differences, zero on the last column / row. */
void orc_forward_gradient(const float *f, float *fx, float *fy, int nx, int ny) {
    for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
            const size_t p = (size_t)y * nx + x;
            fx[p] = (x < nx - 1) ? f[p + 1] - f[p] : 0.0f;
            fy[p] = (y < ny - 1) ? f[p + nx] - f[p] : 0.0f;
        }
}

/* First index of the largest / smallest |x| (BLAS isamax / isamin). */
static size_t first_absmax(const float *x, int n) {
    size_t b = 0;
    float bv = -1.0f;
    for (int i = 0; i < n; i++)
        if (fabsf(x[i]) > bv) { bv = fabsf(x[i]); b = (size_t)i; }
    return b;
}
static size_t first_absmin(const float *x, int n) {
    size_t b = 0;
    float bv = INFINITY;
    for (int i = 0; i < n; i++)
        if (fabsf(x[i]) < bv) { bv = fabsf(x[i]); b = (size_t)i; }
    return b;
}

/* src/tvl1/sequential/tvl1.cpp:302-329: joint range of both frames (chosen by
 * |x| as the BLAS calls do), then 255*(I-min)/(max-min) in double. */
void orc_normalize(float *I0, float *I1, int n) {
    const float a0 = I0[first_absmax(I0, n)], a1 = I1[first_absmax(I1, n)];
    const float b0 = I0[first_absmin(I0, n)], b1 = I1[first_absmin(I1, n)];
    const float mx = (a0 < a1) ? a1 : a0;
    const float mn = (b1 < b0) ? b1 : b0;
    const float den = mx - mn;
    if (den <= 0) return;
    for (int i = 0; i < n; i++) {
        I0[i] = (float)(255.0 * (I0[i] - mn) / den);
        I1[i] = (float)(255.0 * (I1[i] - mn) / den);
    }
}

/* tvl1.cpp:42-43: N = 1 + log(hypot(w,h)/16)/log(1/zfactor), capped. */
int orc_tvl1_nscales(int w, int h, int nscales, float zfactor) {
    const float N = (float)(1 + log(hypot((double)w, (double)h) / 16.0) / logf(1 / zfactor));
    return (N < nscales) ? (int)N : nscales;
}

double orc_tvl1_energy(const float *u1, const float *u2, const float *I1wx,
                       const float *I1wy, const float *rho_c, int nx, int ny, float lambda) {
    double tv = 0.0, data = 0.0;
    for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
            const size_t p = (size_t)y * nx + x;
            const double f1x = (x < nx - 1) ? (double)(u1[p + 1] - u1[p]) : 0.0;
            const double f1y = (y < ny - 1) ? (double)(u1[p + nx] - u1[p]) : 0.0;
            const double f2x = (x < nx - 1) ? (double)(u2[p + 1] - u2[p]) : 0.0;
            const double f2y = (y < ny - 1) ? (double)(u2[p + nx] - u2[p]) : 0.0;
            tv += sqrt(f1x * f1x + f1y * f1y) + sqrt(f2x * f2x + f2y * f2y);
            const float rho = rho_c[p] + (I1wx[p] * u1[p] + I1wy[p] * u2[p]);
            data += fabs((double)rho);
        }
    return tv + (double)lambda * data;
}

/* tvl1.cpp:182-294, one pyramid level. */
void orc_dual_tvl1(const float *I0, const float *I1, float *u1, float *u2, int nx, int ny,
                   const orc_tvl1_params *prm, float *p_out, int *iters, double *energy) {
    const size_t n = (size_t)nx * ny;
    const float l_t = prm->lambda * prm->theta;
    const float taut = prm->tau / prm->theta;
    const float eps2 = prm->epsilon * prm->epsilon;
    float *I1x = falloc(n), *I1y = falloc(n), *I1w = falloc(n), *I1wx = falloc(n),
          *I1wy = falloc(n), *rho_c = falloc(n), *grad = falloc(n), *v1 = falloc(n),
          *v2 = falloc(n), *p11 = falloc(n), *p12 = falloc(n), *p21 = falloc(n),
          *p22 = falloc(n), *d1 = falloc(n), *d2 = falloc(n), *fx1 = falloc(n),
          *fy1 = falloc(n), *fx2 = falloc(n), *fy2 = falloc(n);

    orc_centered_gradient(I1, I1x, I1y, nx, ny);
    for (int w = 0; w < prm->warps; w++) {
        orc_bicubic_warp(I1, u1, u2, I1w, nx, ny, 1);
        orc_bicubic_warp(I1x, u1, u2, I1wx, nx, ny, 1);
        orc_bicubic_warp(I1y, u1, u2, I1wy, nx, ny, 1);
        for (size_t i = 0; i < n; i++) {
            grad[i] = (I1wx[i] * I1wx[i]) + (I1wy[i] * I1wy[i]);
            rho_c[i] = (I1w[i] - I1wx[i] * u1[i] - I1wy[i] * u2[i] - I0[i]);
        }
        int it = 0;
        float error = INFINITY;
        while (error > eps2 && it < prm->max_iterations) {
            it++;
            /* thresholding step TH (tvl1.cpp:221-245) */
            for (size_t i = 0; i < n; i++) {
                const float rho = rho_c[i] + (I1wx[i] * u1[i] + I1wy[i] * u2[i]);
                const float fi = -rho / grad[i];
                const int below = !(rho >= -l_t * grad[i]);
                const int above = rho > l_t * grad[i];
                const int flat = grad[i] < 1E-10f;
                float a1, a2;
                if (below) {
                    a1 = l_t * I1wx[i];
                    a2 = l_t * I1wy[i];
                } else if (above) {
                    a1 = -l_t * I1wx[i];
                    a2 = -l_t * I1wy[i];
                } else if (flat) {
                    a1 = a2 = 0.0f;
                } else {
                    a1 = fi * I1wx[i];
                    a2 = fi * I1wy[i];
                }
                v1[i] = u1[i] + a1;
                v2[i] = u2[i] + a2;
            }
            orc_divergence(p11, p12, d1, nx, ny);
            orc_divergence(p21, p22, d2, nx, ny);
            /* u update and squared change (tvl1.cpp:252-265) */
            float errf = 0.0f;
            double errd = 0.0;
            for (size_t i = 0; i < n; i++) {
                const float u1k = u1[i], u2k = u2[i];
                u1[i] = v1[i] + prm->theta * d1[i];
                u2[i] = v2[i] + prm->theta * d2[i];
                const float term = (u1[i] - u1k) * (u1[i] - u1k) + (u2[i] - u2k) * (u2[i] - u2k);
                errf += term;
                errd += term;
            }
            error = prm->error_mode ? (float)errd : errf;
            error /= (float)n;
            if (energy)
                energy[(size_t)w * prm->max_iterations + (it - 1)] =
                    orc_tvl1_energy(u1, u2, I1wx, I1wy, rho_c, nx, ny, prm->lambda);
            /* dual update (tvl1.cpp:268-291) */
            orc_forward_gradient(u1, fx1, fy1, nx, ny);
            orc_forward_gradient(u2, fx2, fy2, nx, ny);
            for (size_t i = 0; i < n; i++) {
                const float g1 = 1.0f + taut * hypotf(fx1[i], fy1[i]);
                const float g2 = 1.0f + taut * hypotf(fx2[i], fy2[i]);
                float t;
                t = taut * fx1[i]; p11[i] = t + p11[i];
                t = taut * fy1[i]; p12[i] = t + p12[i];
                t = taut * fx2[i]; p21[i] = t + p21[i];
                t = taut * fy2[i]; p22[i] = t + p22[i];
                p11[i] = p11[i] / g1;
                p12[i] = p12[i] / g1;
                p21[i] = p21[i] / g2;
                p22[i] = p22[i] / g2;
            }
        }
        if (iters) iters[w] = it;
    }
    if (p_out) {
        memcpy(p_out, p11, n * sizeof(float));
        memcpy(p_out + n, p12, n * sizeof(float));
        memcpy(p_out + 2 * n, p21, n * sizeof(float));
        memcpy(p_out + 3 * n, p22, n * sizeof(float));
    }
    float *bufs[] = {I1x, I1y, I1w, I1wx, I1wy, rho_c, grad, v1, v2, p11,
                     p12, p21, p22, d1, d2, fx1, fy1, fx2, fy2};
    for (size_t k = 0; k < sizeof(bufs) / sizeof(bufs[0]); k++) free(bufs[k]);
}

/* tvl1.cpp:129-175, from float frames. */
int orc_tvl1(const float *I0, const float *I1, int w, int h, const orc_tvl1_params *prm,
             float *u, float *v, orc_tvl1_trace *trace) {
    const int ns = orc_tvl1_nscales(w, h, prm->nscales, prm->zfactor);
    if (ns < 1 || ns > 32) return -1;
    float *I0s[32], *I1s[32], *u1s[32], *u2s[32];
    int nx[32], ny[32];
    nx[0] = w;
    ny[0] = h;
    for (int s = 1; s < ns; s++) orc_zoom_size(nx[s - 1], ny[s - 1], &nx[s], &ny[s], prm->zfactor);
    for (int s = 0; s < ns; s++) {
        const size_t n = (size_t)nx[s] * ny[s];
        I0s[s] = falloc(n); I1s[s] = falloc(n); u1s[s] = falloc(n); u2s[s] = falloc(n);
    }
    int rc = 0;
    memcpy(I0s[0], I0, sizeof(float) * (size_t)w * h);
    memcpy(I1s[0], I1, sizeof(float) * (size_t)w * h);
    orc_normalize(I0s[0], I1s[0], w * h);
    if (orc_gaussian(I0s[0], w, h, 0.8f) || orc_gaussian(I1s[0], w, h, 0.8f)) rc = -1;
    for (int s = 1; s < ns && rc == 0; s++) {
        if (orc_zoom_out(I0s[s - 1], I0s[s], nx[s - 1], ny[s - 1], prm->zfactor) ||
            orc_zoom_out(I1s[s - 1], I1s[s], nx[s - 1], ny[s - 1], prm->zfactor))
            rc = -1;
    }
    if (rc == 0) {
        const float inv = 1 / prm->zfactor;
        for (int s = ns - 1; s >= 0; s--) {
            int *it = trace && trace->iterations ? trace->iterations + (size_t)s * prm->warps : NULL;
            double *en = trace && trace->energy
                             ? trace->energy + (size_t)s * prm->warps * prm->max_iterations
                             : NULL;
            orc_dual_tvl1(I0s[s], I1s[s], u1s[s], u2s[s], nx[s], ny[s], prm, NULL, it, en);
            if (s == 0) break;
            orc_zoom_in(u1s[s], u1s[s - 1], nx[s], ny[s], nx[s - 1], ny[s - 1]);
            orc_zoom_in(u2s[s], u2s[s - 1], nx[s], ny[s], nx[s - 1], ny[s - 1]);
            const size_t n = (size_t)nx[s - 1] * ny[s - 1];
            for (size_t i = 0; i < n; i++) {
                u1s[s - 1][i] = inv * u1s[s - 1][i];
                u2s[s - 1][i] = inv * u2s[s - 1][i];
            }
        }
        memcpy(u, u1s[0], sizeof(float) * (size_t)w * h);
        memcpy(v, u2s[0], sizeof(float) * (size_t)w * h);
    }
    for (int s = 0; s < ns; s++) { free(I0s[s]); free(I1s[s]); free(u1s[s]); free(u2s[s]); }
    return rc == 0 ? ns : -1;
}

/* ===================================================================== */
/* Horn-Schunck (CPU restatement of src/hs/cuda)                          */
/* ===================================================================== */

/* 2x2 box average to (w/2, h/2), src/hs/cuda/kernels/downscaleKernel.cuh:27-29.
 * Deviation: every output sample is written (the kernel's guard skips the last
 * row and column, :32). */
void orc_hs_downscale(const float *src, int w, int h, float *dst) {
    const int nw = w / 2, nh = h / 2;
    for (int y = 0; y < nh; y++)
        for (int x = 0; x < nw; x++) {
            const size_t a = (size_t)(2 * y) * w + 2 * x;
            dst[(size_t)y * nw + x] = 0.25f * (src[a] + src[a + w] + src[a + 1] + src[a + w + 1]);
        }
}

/* Bilinear sample with clamp-to-edge taps at (x, y) in pixel units; the
 * coordinate is first limited to [-1, n] so the integer part cannot overflow. */
static inline float bilinear_clamped(const float *src, int w, int h, float xf, float yf) {
    xf = fminf(fmaxf(xf, -1.0f), (float)w);
    yf = fminf(fmaxf(yf, -1.0f), (float)h);
    const float x0f = floorf(xf), y0f = floorf(yf);
    const float fx = xf - x0f, fy = yf - y0f;
    const int x0 = (int)x0f, y0 = (int)y0f;
    const int xa = imin(imax(x0, 0), w - 1), xb = imin(imax(x0 + 1, 0), w - 1);
    const int ya = imin(imax(y0, 0), h - 1), yb = imin(imax(y0 + 1, 0), h - 1);
    const float v00 = src[(size_t)ya * w + xa], v10 = src[(size_t)ya * w + xb];
    const float v01 = src[(size_t)yb * w + xa], v11 = src[(size_t)yb * w + xb];
    const float gx = 1.0f - fx, gy = 1.0f - fy;
    const float top = gx * v00 + fx * v10;
    const float bot = gx * v01 + fx * v11;
    return gy * top + fy * bot;
}

/* out(x,y) = src(x+u, y+v), bilinear, clamp-to-edge.  This is what
 * src/hs/cuda/kernels/warpingKernel.cuh:28-44 is written to do with a
 * filtering texture; the literal index arithmetic there (:38-40) indexes the
 * array with normalised coordinates, which this restatement does not follow. */
void orc_bilinear_warp(const float *src, const float *u, const float *v, int w, int h,
                       float *out) {
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            const size_t p = (size_t)y * w + x;
            out[p] = bilinear_clamped(src, w, h, (float)x + u[p], (float)y + v[p]);
        }
}

void orc_hs_warp(const float *src, const float *u, const float *v, int w, int h, float *out) {
    orc_bilinear_warp(src, u, v, w, h, out);
}

/* (1,-8,0,8,-1)/12 derivative of one image along a line of clamped indices,
 * accumulated in the kernel's order (derivativesKernel.cuh:42-46). */
static inline float deriv5(float a_m2, float a_m1, float a_p1, float a_p2) {
    float t = a_m2;
    t -= a_m1 * 8.0f;
    t += a_p1 * 8.0f;
    t -= a_p2;
    t /= 12.0f;
    return t;
}

/* derivativesKernel.cuh:29-73.  Deviation: indices are clamped everywhere and
 * every pixel is written (the kernel reads before the start for x,y < 2 and
 * leaves the last two rows and columns unwritten). */
void orc_hs_derivatives(const float *I0, const float *I1w, int w, int h, float *Ix, float *Iy,
                        float *Iz) {
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            const size_t row = (size_t)y * w;
            const int xm2 = imax(x - 2, 0), xm1 = imax(x - 1, 0);
            const int xp1 = imin(x + 1, w - 1), xp2 = imin(x + 2, w - 1);
            const int ym2 = imax(y - 2, 0), ym1 = imax(y - 1, 0);
            const int yp1 = imin(y + 1, h - 1), yp2 = imin(y + 2, h - 1);
            float t0 = deriv5(I0[row + xm2], I0[row + xm1], I0[row + xp1], I0[row + xp2]);
            float t1 = deriv5(I1w[row + xm2], I1w[row + xm1], I1w[row + xp1], I1w[row + xp2]);
            Ix[row + x] = (t0 + t1) * 0.5f;
            Iz[row + x] = I1w[row + x] - I0[row + x];
            t0 = deriv5(I0[(size_t)ym2 * w + x], I0[(size_t)ym1 * w + x], I0[(size_t)yp1 * w + x],
                        I0[(size_t)yp2 * w + x]);
            t1 = deriv5(I1w[(size_t)ym2 * w + x], I1w[(size_t)ym1 * w + x],
                        I1w[(size_t)yp1 * w + x], I1w[(size_t)yp2 * w + x]);
            Iy[row + x] = (t0 + t1) * 0.5f;
        }
}

/* One Jacobi sweep, src/hs/cuda/kernels/solverKernel.cuh:41-153: mean of the
 * four clamped neighbours (left, right, next row, previous row, in that
 * order), then the point update with alpha added as given (not squared). */
void orc_hs_jacobi(const float *du0, const float *dv0, const float *Ix, const float *Iy,
                   const float *Iz, int w, int h, float alpha, float *du1, float *dv1) {
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            const size_t p = (size_t)y * w + x;
            const size_t l = (size_t)y * w + imax(x - 1, 0), r = (size_t)y * w + imin(x + 1, w - 1);
            const size_t up = (size_t)imin(y + 1, h - 1) * w + x, dn = (size_t)imax(y - 1, 0) * w + x;
            const float su = (du0[l] + du0[r] + du0[up] + du0[dn]) * 0.25f;
            const float sv = (dv0[l] + dv0[r] + dv0[up] + dv0[dn]) * 0.25f;
            const float frac = (Ix[p] * su + Iy[p] * sv + Iz[p]) / (Ix[p] * Ix[p] + Iy[p] * Iy[p] + alpha);
            du1[p] = su - Ix[p] * frac;
            dv1[p] = sv - Iy[p] * frac;
        }
}

/* Flow upsampling to (nw, nh): bilinear, clamp-to-edge, sample centres aligned
 * ((x+0.5)*w/nw - 0.5), times `scale`.  This is the filtering-texture
 * upscale that src/hs/cuda/kernels/upscaleKernel.cuh:26-40 is written for; its
 * literal point sample (with a negative index at x=0) is not followed. */
void orc_upscale(const float *src, int w, int h, int nw, int nh, float scale, float *dst) {
    const float rx = (float)w / (float)nw, ry = (float)h / (float)nh;
    for (int y = 0; y < nh; y++)
        for (int x = 0; x < nw; x++) {
            const float sx = ((float)x + 0.5f) * rx - 0.5f;
            const float sy = ((float)y + 0.5f) * ry - 0.5f;
            dst[(size_t)y * nw + x] = bilinear_clamped(src, w, h, sx, sy) * scale;
        }
}

/* src/hs/cuda/flow.cu:112-208.  The finest level is nlevels-1. */
int orc_hs(const float *I0, const float *I1, int w, int h, float alpha, int nlevels, int nwarp,
           int nsolver, float *u, float *v) {
    if (nlevels < 1 || nlevels > 16 || w < 1 || h < 1) return -1;
    int W[16], H[16];
    float *P0[16], *P1[16];
    W[nlevels - 1] = w;
    H[nlevels - 1] = h;
    for (int l = nlevels - 1; l > 0; l--) {
        W[l - 1] = W[l] / 2;
        H[l - 1] = H[l] / 2;
        if (W[l - 1] < 1 || H[l - 1] < 1) return -1;
    }
    for (int l = 0; l < nlevels; l++) {
        P0[l] = falloc((size_t)W[l] * H[l]);
        P1[l] = falloc((size_t)W[l] * H[l]);
    }
    memcpy(P0[nlevels - 1], I0, sizeof(float) * (size_t)w * h);
    memcpy(P1[nlevels - 1], I1, sizeof(float) * (size_t)w * h);
    for (int l = nlevels - 1; l > 0; l--) {
        orc_hs_downscale(P0[l], W[l], H[l], P0[l - 1]);
        orc_hs_downscale(P1[l], W[l], H[l], P1[l - 1]);
    }
    const size_t N = (size_t)w * h;
    float *cu = falloc(N), *cv = falloc(N), *nu = falloc(N), *nv = falloc(N), *tmp = falloc(N);
    float *Ix = falloc(N), *Iy = falloc(N), *Iz = falloc(N);
    float *du0 = falloc(N), *dv0 = falloc(N), *du1 = falloc(N), *dv1 = falloc(N);
    for (int l = 0; l < nlevels; l++) {
        const int lw = W[l], lh = H[l];
        const size_t n = (size_t)lw * lh;
        for (int wi = 0; wi < nwarp; wi++) {
            memset(du0, 0, n * sizeof(float));
            memset(dv0, 0, n * sizeof(float));
            orc_hs_warp(P1[l], cu, cv, lw, lh, tmp);
            orc_hs_derivatives(P0[l], tmp, lw, lh, Ix, Iy, Iz);
            for (int it = 0; it < nsolver; it++) {
                orc_hs_jacobi(du0, dv0, Ix, Iy, Iz, lw, lh, alpha, du1, dv1);
                float *t = du0; du0 = du1; du1 = t;
                t = dv0; dv0 = dv1; dv1 = t;
            }
            for (size_t i = 0; i < n; i++) {
                cu[i] = cu[i] + du0[i];
                cv[i] = cv[i] + dv0[i];
            }
        }
        if (l != nlevels - 1) {
            const float sx = (float)W[l + 1] / (float)W[l];
            const float sy = (float)H[l + 1] / (float)H[l];
            orc_upscale(cu, lw, lh, W[l + 1], H[l + 1], sx, nu);
            orc_upscale(cv, lw, lh, W[l + 1], H[l + 1], sy, nv);
            float *t = cu; cu = nu; nu = t;
            t = cv; cv = nv; nv = t;
        }
    }
    memcpy(u, cu, N * sizeof(float));
    memcpy(v, cv, N * sizeof(float));
    float *bufs[] = {cu, cv, nu, nv, tmp, Ix, Iy, Iz, du0, dv0, du1, dv1};
    for (size_t k = 0; k < sizeof(bufs) / sizeof(bufs[0]); k++) free(bufs[k]);
    for (int l = 0; l < nlevels; l++) { free(P0[l]); free(P1[l]); }
    return 0;
}

/* ===================================================================== */
/* Lucas-Kanade (CPU restatement of src/lk/cuda)                          */
/* ===================================================================== */

/* Central-difference FIR taps, src/lk/cuda/lucaskanade.cu:79-161. Returns -1
 * for sizes the reference does not define. */
int orc_lk_filters(int spac_size, int temp_size, float *fs, float *ft) {
    static const float s1[] = {1.0f};
    static const float s3[] = {-1.0f / 2.0f, 0.0f, 1.0f / 2.0f};
    static const float s5[] = {1.0f / 12.0f, -2.0f / 3.0f, 0.0f, 2.0f / 3.0f, -1.0f / 12.0f};
    static const float s7[] = {-1.0f / 60.0f, 3.0f / 20.0f, -3.0f / 4.0f, 0.0f,
                               3.0f / 4.0f,   -3.0f / 20.0f, 1.0f / 60.0f};
    static const float s9[] = {1.0f / 280.0f, -4.0f / 105.0f, 1.0f / 5.0f, -4.0f / 5.0f, 0.0f,
                               4.0f / 5.0f,   -1.0f / 5.0f,   4.0f / 105.0f, -1.0f / 280.0f};
    static const float t2[] = {-1.0f, 1.0f};
    const float *S = NULL, *T = NULL;
    switch (spac_size) {
        case 1: S = s1; break;
        case 3: S = s3; break;
        case 5: S = s5; break;
        case 7: S = s7; break;
        case 9: S = s9; break;
        default: return -1;
    }
    switch (temp_size) {
        case 1: T = s1; break;
        case 2: T = t2; break;
        case 3: T = s3; break;
        case 5: T = s5; break;
        case 7: T = s7; break;
        case 9: T = s9; break;
        default: return -1;
    }
    if (fs) memcpy(fs, S, sizeof(float) * spac_size);
    if (ft) memcpy(ft, T, sizeof(float) * temp_size);
    return 0;
}

/* Zero-padded FIR along x or y of a float image (src/lk/cuda/kernels/kernels.cu:
 * 44-121: taps that fall outside are dropped, accumulation in tap order).
 * Deviation: the y pass tests the bottom border against the height (the
 * kernel tests against the width, :106). */
static void conv_x(const float *f, float *out, int nx, int ny, const float *k, int ks) {
    const int c = (ks - 1) / 2;
    for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
            float acc = 0.0f;
            for (int t = 0; t < ks; t++) {
                const int xx = x + t - c;
                if (xx < 0 || xx >= nx) continue;
                acc += f[(size_t)y * nx + xx] * k[t];
            }
            out[(size_t)y * nx + x] = acc;
        }
}
static void conv_y(const float *f, float *out, int nx, int ny, const float *k, int ks) {
    const int c = (ks - 1) / 2;
    for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
            float acc = 0.0f;
            for (int t = 0; t < ks; t++) {
                const int yy = y + t - c;
                if (yy < 0 || yy >= ny) continue;
                acc += f[(size_t)yy * nx + x] * k[t];
            }
            out[(size_t)y * nx + x] = acc;
        }
}

/* 5 window sums in row-major order and the closed-form 2x2 solve
 * (kernels.cu:134-181).  Deviation: pixels closer than the window radius to
 * the border are written as 0 (the kernel leaves them unwritten). */
static void lk_solve(const float *Ix, const float *Iy, const float *It, int nx, int ny,
                     int window, float *Vx, float *Vy) {
    const int c = (window - 1) / 2;
    for (int i = 0; i < ny; i++)
        for (int j = 0; j < nx; j++) {
            const size_t o = (size_t)i * nx + j;
            Vx[o] = 0.0f;
            Vy[o] = 0.0f;
            if (!(i >= c && j >= c && i < ny - c && j < nx - c)) continue;
            float sxx = 0.0f, sxy = 0.0f, syy = 0.0f, sxt = 0.0f, syt = 0.0f;
            for (int ii = -c; ii <= c; ii++)
                for (int jj = -c; jj <= c; jj++) {
                    const size_t q = (size_t)(i + ii) * nx + (j + jj);
                    sxx += Ix[q] * Ix[q];
                    sxy += Ix[q] * Iy[q];
                    syy += Iy[q] * Iy[q];
                    sxt += Ix[q] * It[q];
                    syt += Iy[q] * It[q];
                }
            const float det = (sxx * syy - sxy * sxy);
            if (det != 0.0f) {
                Vx[o] = 1.0f / det * (syy * (-sxt) + (-sxy) * (-syt));
                Vy[o] = 1.0f / det * ((-sxy) * (-sxt) + sxx * (-syt));
            }
        }
}

int orc_lk(const uint8_t *const *frames, int nx, int ny, int spac_size, int temp_size,
           int window, int iframe, float *Vx, float *Vy) {
    float fs[9], ft[9];
    if (orc_lk_filters(spac_size, temp_size, fs, ft) || window < 1 || (window & 1) == 0)
        return -1;
    const size_t n = (size_t)nx * ny;
    float *It = falloc(n), *Ix = falloc(n), *Iy = falloc(n), *old = falloc(n);
    /* temporal FIR over the ring, oldest slot first (kernels.cu:14-30) */
    for (size_t p = 0; p < n; p++) It[p] = 0.0f;
    for (int fr = 0; fr < temp_size; fr++) {
        const uint8_t *im = frames[(fr + iframe + 1) % temp_size];
        for (size_t p = 0; p < n; p++) It[p] += ft[fr] * (float)im[p];
    }
    /* spatial derivatives of the oldest frame in the ring (lucaskanade.cu:56) */
    const uint8_t *f0 = frames[(iframe + 1) % temp_size];
    for (size_t p = 0; p < n; p++) old[p] = (float)f0[p];
    conv_x(old, Ix, nx, ny, fs, spac_size);
    conv_y(old, Iy, nx, ny, fs, spac_size);
    lk_solve(Ix, Iy, It, nx, ny, window, Vx, Vy);
    free(It); free(Ix); free(Iy); free(old);
    return 0;
}

/* Two float frames, temporal taps (-1, 1): It = 0 + (-1)*I0 + 1*I1. */
static void temporal2(const float *I0, const float *I1, float *It, size_t n) {
    for (size_t p = 0; p < n; p++) {
        float acc = 0.0f;
        acc += -1.0f * I0[p];
        acc += 1.0f * I1[p];
        It[p] = acc;
    }
}

int orc_lk_f32(const float *I0, const float *I1, int nx, int ny, int spac_size, int window,
               float *Vx, float *Vy) {
    float fs[9];
    if (orc_lk_filters(spac_size, 2, fs, NULL) || window < 1 || (window & 1) == 0) return -1;
    const size_t n = (size_t)nx * ny;
    float *It = falloc(n), *Ix = falloc(n), *Iy = falloc(n);
    temporal2(I0, I1, It, n);
    conv_x(I0, Ix, nx, ny, fs, spac_size);
    conv_y(I0, Iy, nx, ny, fs, spac_size);
    lk_solve(Ix, Iy, It, nx, ny, window, Vx, Vy);
    free(It); free(Ix); free(Iy);
    return 0;
}

/* Pyramidal, iterated LK (no reference counterpart; composed from the steps
 * above).  Pyramid: the TV-L1 zoom_out at factor 0.5 (Gaussian + decimation).
 * Per level, coarse to fine, `iters` times: warp I1 by the current flow
 * (bilinear, clamp-to-edge), It = I1w - I0 by the temporal taps, Ix/Iy of I0,
 * window solve, flow += increment.  Between levels: orc_upscale with the
 * size ratio as scale. */
int orc_pyrlk(const float *I0, const float *I1, int w, int h, int levels, int iters,
              int spac_size, int window, float *u, float *v) {
    float fs[9];
    if (levels < 1 || levels > 16 || orc_lk_filters(spac_size, 2, fs, NULL)) return -1;
    int W[16], H[16];
    float *P0[16], *P1[16];
    W[0] = w;
    H[0] = h;
    for (int l = 1; l < levels; l++) orc_zoom_size(W[l - 1], H[l - 1], &W[l], &H[l], 0.5f);
    for (int l = 0; l < levels; l++) {
        P0[l] = falloc((size_t)W[l] * H[l]);
        P1[l] = falloc((size_t)W[l] * H[l]);
    }
    memcpy(P0[0], I0, sizeof(float) * (size_t)w * h);
    memcpy(P1[0], I1, sizeof(float) * (size_t)w * h);
    int rc = 0;
    for (int l = 1; l < levels && rc == 0; l++)
        if (orc_zoom_out(P0[l - 1], P0[l], W[l - 1], H[l - 1], 0.5f) ||
            orc_zoom_out(P1[l - 1], P1[l], W[l - 1], H[l - 1], 0.5f))
            rc = -1;
    const size_t N = (size_t)w * h;
    float *cu = falloc(N), *cv = falloc(N), *nu = falloc(N), *nv = falloc(N);
    float *I1w = falloc(N), *It = falloc(N), *Ix = falloc(N), *Iy = falloc(N);
    float *du = falloc(N), *dv = falloc(N);
    for (int l = levels - 1; l >= 0 && rc == 0; l--) {
        const int lw = W[l], lh = H[l];
        const size_t n = (size_t)lw * lh;
        conv_x(P0[l], Ix, lw, lh, fs, spac_size);
        conv_y(P0[l], Iy, lw, lh, fs, spac_size);
        for (int r = 0; r < iters; r++) {
            orc_bilinear_warp(P1[l], cu, cv, lw, lh, I1w);
            temporal2(P0[l], I1w, It, n);
            lk_solve(Ix, Iy, It, lw, lh, window, du, dv);
            for (size_t i = 0; i < n; i++) {
                cu[i] = cu[i] + du[i];
                cv[i] = cv[i] + dv[i];
            }
        }
        if (l > 0) {
            const float sx = (float)W[l - 1] / (float)lw;
            const float sy = (float)H[l - 1] / (float)lh;
            orc_upscale(cu, lw, lh, W[l - 1], H[l - 1], sx, nu);
            orc_upscale(cv, lw, lh, W[l - 1], H[l - 1], sy, nv);
            float *t = cu; cu = nu; nu = t;
            t = cv; cv = nv; nv = t;
        }
    }
    if (rc == 0) {
        memcpy(u, cu, N * sizeof(float));
        memcpy(v, cv, N * sizeof(float));
    }
    float *bufs[] = {cu, cv, nu, nv, I1w, It, Ix, Iy, du, dv};
    for (size_t k = 0; k < sizeof(bufs) / sizeof(bufs[0]); k++) free(bufs[k]);
    for (int l = 0; l < levels; l++) { free(P0[l]); free(P1[l]); }
    return rc;
}


/* ===================================================================== flowToColor */
/* main.cpp:93-126.  The reference computes |f| and atan2 in float, scales with
 * OpenCV Mat expressions and converts to 8 bits with saturate_cast (round to
 * nearest even, clamp to 0..255), then converts HSV to BGR with cvtColor.
 * OpenCV is not part of the reference tree; its HSV->BGR conversion is the
 * hexcone model (Smith 1978) with H stored as degrees/2 and S, V scaled to
 * 0..255, restated here in single precision:
 *   h' = H * (6/180), sector = floor(h'), f = h' - sector, s = S/255, v = V/255
 *   p = v(1-s), q = v(1-s f), t = v(1-s(1-f))
 *   (R,G,B) = (v,t,p) (q,v,p) (p,v,t) (p,q,v) (t,p,v) (v,p,q) for sectors 0..5
 *   byte = saturate(255 x).
 * atan2 is taken in double and rounded to float, which equals a correctly
 * rounded atan2f. */
static uint8_t sat_u8(float x) {
    if (!(x == x)) return 0;
    const float r = rintf(x);
    if (r <= 0.0f) return 0;
    if (r >= 255.0f) return 255;
    return (uint8_t)r;
}

void orc_flow_to_color(const float *u, const float *v, int w, int h, uint8_t *bgr) {
    const float hue_scale = (float)(180.0 / 3.14159265358979323846 / 2.0);
    for (size_t i = 0; i < (size_t)w * h; i++) {
        const float fu = u[i], fv = v[i];
        const float mag = sqrtf(fu * fu + fv * fv);
        float m = mag * 10.0f;
        if (m > 255.0f) m = 255.0f;
        const uint8_t V = sat_u8(m);
        const float ang = (float)atan2((double)fv, (double)fu);
        const uint8_t H = sat_u8(ang * hue_scale);
        const float hh = (float)H * (6.0f / 180.0f);
        int sector = (int)floorf(hh);
        float f = hh - (float)sector;
        if (sector < 0 || sector > 5) {
            sector = 0;
            f = 0.0f;
        }
        const float s = 255.0f * (1.0f / 255.0f);
        const float vv = (float)V * (1.0f / 255.0f);
        const float p = vv * (1.0f - s), q = vv * (1.0f - s * f), t = vv * (1.0f - s * (1.0f - f));
        float r, g, b;
        switch (sector) {
            case 0: r = vv; g = t; b = p; break;
            case 1: r = q; g = vv; b = p; break;
            case 2: r = p; g = vv; b = t; break;
            case 3: r = p; g = q; b = vv; break;
            case 4: r = t; g = p; b = vv; break;
            default: r = vv; g = p; b = q; break;
        }
        bgr[3 * i + 0] = sat_u8(b * 255.0f);
        bgr[3 * i + 1] = sat_u8(g * 255.0f);
        bgr[3 * i + 2] = sat_u8(r * 255.0f);
    }
}
