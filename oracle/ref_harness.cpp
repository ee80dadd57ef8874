/*
 * C entry points around the reference's sequential TV-L1, compiled from the
 * reference sources in place (src/tvl1/sequential/{tvl1,mask/mask,zoom/zoom,
 * bicubic_interpolation/bicubic_interpolation}.cpp) into oracle/_ref.
 *
 * Test infrastructure only: the parity tests, the golden-fixture script and the
 * CPU-baseline leg of bench.py load this library as the checker.  Nothing in the
 * product links it.
 *
 * The reference object has a destructor double free (tvl1.cpp:132 aliases
 * _u1s[0] to _u and _u2s[0] into its second half; ~TV_L1 deletes all three,
 * tvl1.cpp:82 and :87-88).  release_object() points both at fresh allocations
 * before deleting, so the object can be destroyed without touching the
 * reference code.
 */
#include <cmath>
#include <cstring>
#include <cstdint>
#include <cstdlib>

#include "ref_shim/tvl1_decl.hpp"

/* The reference declares these in headers that also declare a static
 * function; re-declaring the public ones here keeps this file independent. */
void divergence(const float *v1, const float *v2, float *div, const int nx, const int ny);
void forward_gradient(const float *f, float *fx, float *fy, const int nx, const int ny);
void centered_gradient(const float *input, float *dx, float *dy, const int nx, const int ny);
void gaussian(float *I, const int xdim, const int ydim, const double sigma, float *buffer);
void zoom_out(const float *I, float *Iout, const int nx, const int ny, const float factor,
              float *Is, float *gaussBuffer);
void zoom_in(const float *I, float *Iout, int nx, int ny, int nxx, int nyy);
float bicubic_interpolation_at(const float *input, const float uu, const float vv,
                               const int nx, const int ny, bool border_out);
void bicubic_interpolation_warp(const float *input, const float *u, const float *v,
                                float *output, const int nx, const int ny, bool border_out);

std::size_t MAX_ITERATIONS = 300;

namespace {

struct Cached {
    TV_L1 *obj = nullptr;
    int w = 0, h = 0, nscales = 0, warps = 0;
    float tau = 0, lambda = 0, theta = 0, zfactor = 0, eps = 0;
};
Cached g_cache;

void release_object(TV_L1 *t) {
    if (!t) return;
    if (t->_nscales > 0 && t->_u1s[0] == t->_u) {
        t->_u1s[0] = new float[1];
        t->_u2s[0] = new float[1]; /* pointed into the middle of _u */
    }
    delete t;
}

TV_L1 *get_object(int w, int h, float tau, float lambda, float theta, int nscales,
                  float zfactor, int warps, float eps) {
    Cached &c = g_cache;
    if (c.obj && c.w == w && c.h == h && c.tau == tau && c.lambda == lambda &&
        c.theta == theta && c.nscales == nscales && c.zfactor == zfactor &&
        c.warps == warps && c.eps == eps)
        return c.obj;
    release_object(c.obj);
    c.obj = new TV_L1(w, h, tau, lambda, theta, nscales, zfactor, warps, eps);
    c.w = w; c.h = h; c.tau = tau; c.lambda = lambda; c.theta = theta;
    c.nscales = nscales; c.zfactor = zfactor; c.warps = warps; c.eps = eps;
    return c.obj;
}

/* gaussian() terminates the process when the window exceeds the width
 * (mask.cpp:231-234); callers are checked first. */
int gaussian_window(double sigma) { return (int)(5 * sigma) + 1; }

}  // namespace

extern "C" {

void ref_set_max_iterations(long long n) { MAX_ITERATIONS = (std::size_t)n; }
long long ref_get_max_iterations(void) { return (long long)MAX_ITERATIONS; }

/* Number of scales the reference constructor picks (tvl1.cpp:42-43). */
int ref_tvl1_nscales(int w, int h, int nscales, float zfactor) {
    TV_L1 *t = get_object(w, h, 0.25f, 0.15f, 0.3f, nscales, zfactor, 5, 0.01f);
    return t->_nscales;
}

/* Full multiscale solve (tvl1.cpp:129-175).  u, v: w*h each. Returns nscales. */
int ref_tvl1_run(const uint8_t *I0, const uint8_t *I1, int w, int h, float tau,
                 float lambda, float theta, int nscales, float zfactor, int warps,
                 float eps, float *u, float *v) {
    TV_L1 *t = get_object(w, h, tau, lambda, theta, nscales, zfactor, warps, eps);
    /* every level must admit both Gaussian windows (sigma 0.8 at level 0, the
     * zoom sigma on every level it is applied to) */
    int nx = w, ny = h;
    const float zs = (float)(0.6f * std::sqrt(1.0 / (zfactor * zfactor) - 1.0));
    if (gaussian_window(0.8f) > nx) return -1;
    for (int s = 1; s < t->_nscales; s++) {
        if (gaussian_window(zs) > nx) return -1;
        nx = (int)((float)nx * zfactor + 0.5);
        ny = (int)((float)ny * zfactor + 0.5);
    }
    t->runDualTVL1Multiscale(const_cast<uint8_t *>(I0), const_cast<uint8_t *>(I1));
    const float *U = t->getU();
    std::memcpy(u, U, sizeof(float) * (size_t)w * h);
    std::memcpy(v, U + (size_t)w * h, sizeof(float) * (size_t)w * h);
    return t->_nscales;
}

/* Pyramid images after a run (level s, nx[s]*ny[s] floats each). */
int ref_tvl1_level(int s, float *I0s, float *I1s, int *nx, int *ny) {
    TV_L1 *t = g_cache.obj;
    if (!t || s < 0 || s >= t->_nscales) return -1;
    *nx = t->_nx[s];
    *ny = t->_ny[s];
    const size_t n = (size_t)t->_nx[s] * t->_ny[s];
    if (I0s) std::memcpy(I0s, t->_I0s[s], n * sizeof(float));
    if (I1s) std::memcpy(I1s, t->_I1s[s], n * sizeof(float));
    return 0;
}

/* One pyramid level (tvl1.cpp:182-294) on caller data.  u1, u2 are updated in
 * place; p (optional, 4*nx*ny) receives p11|p12|p21|p22 after the solve. */
void ref_dual_tvl1(const float *I0, const float *I1, float *u1, float *u2, int nx, int ny,
                   float tau, float lambda, float theta, int warps, float eps, float *p) {
    TV_L1 *t = new TV_L1(nx, ny, tau, lambda, theta, 1, 0.5f, warps, eps);
    t->dualTVL1(I0, I1, u1, u2, nx, ny);
    const size_t n = (size_t)nx * ny;
    if (p) {
        std::memcpy(p, t->_p11, n * sizeof(float));
        std::memcpy(p + n, t->_p12, n * sizeof(float));
        std::memcpy(p + 2 * n, t->_p21, n * sizeof(float));
        std::memcpy(p + 3 * n, t->_p22, n * sizeof(float));
    }
    delete t; /* never ran runDualTVL1Multiscale, so no aliasing */
}

void ref_normalize(const float *I0, const float *I1, float *I0n, float *I1n, int size) {
    TV_L1 t(4, 4);
    t.image_normalization(I0, I1, I0n, I1n, size);
}

int ref_gaussian(float *I, int xdim, int ydim, double sigma) {
    const int size = gaussian_window(sigma);
    if (size > xdim) return -1;
    float *buf = new float[(size_t)(xdim > ydim ? xdim : ydim) + 2 * size + 8];
    gaussian(I, xdim, ydim, sigma, buf);
    delete[] buf;
    return 0;
}

int ref_zoom_out(const float *I, float *Iout, int nx, int ny, float factor) {
    const float zs = (float)(0.6f * std::sqrt(1.0 / (factor * factor) - 1.0));
    if (gaussian_window(zs) > nx) return -1;
    float *Is = new float[(size_t)nx * ny];
    float *buf = new float[(size_t)(nx > ny ? nx : ny) + 64];
    zoom_out(I, Iout, nx, ny, factor, Is, buf);
    delete[] Is;
    delete[] buf;
    return 0;
}

void ref_zoom_in(const float *I, float *Iout, int nx, int ny, int nxx, int nyy) {
    zoom_in(I, Iout, nx, ny, nxx, nyy);
}

float ref_bicubic_at(const float *input, float uu, float vv, int nx, int ny, int border_out) {
    return bicubic_interpolation_at(input, uu, vv, nx, ny, border_out != 0);
}

void ref_bicubic_warp(const float *input, const float *u, const float *v, float *out, int nx,
                      int ny, int border_out) {
    bicubic_interpolation_warp(input, u, v, out, nx, ny, border_out != 0);
}

void ref_centered_gradient(const float *in, float *dx, float *dy, int nx, int ny) {
    centered_gradient(in, dx, dy, nx, ny);
}

void ref_divergence(const float *v1, const float *v2, float *div, int nx, int ny) {
    divergence(v1, v2, div, nx, ny);
}

void ref_forward_gradient(const float *f, float *fx, float *fy, int nx, int ny) {
    forward_gradient(f, fx, fy, nx, ny);
}

}  // extern "C"
