/*
 * CPU oracle for the three dense optical-flow solvers (TV-L1, Horn-Schunck,
 * Lucas-Kanade).  TEST INFRASTRUCTURE: only tests/, the smoke check and the
 * CPU-baseline leg of bench.py load it, as the checker.  The product never
 * links or calls it.
 *
 * TV-L1 restates the reference's sequential C++ path
 * (src/tvl1/sequential/{tvl1,mask/mask,zoom/zoom,bicubic_interpolation/
 * bicubic_interpolation}.cpp) operation for operation, including its double
 * precision literals, so that with the reference's single-threaded error sum
 * it is bit-identical to the reference compiled in oracle/_ref.
 *
 * HS and LK have no CPU code in the reference; they restate the CUDA kernels
 * of the src/hs/cuda/kernels headers and src/lk/cuda/kernels/kernels.cu with the
 * deviations listed at each function (the literal kernels read out of bounds
 * or leave outputs unwritten).
 *
 * Arithmetic: IEEE single/double exactly as written, no fused multiply-add
 * (built with -ffp-contract=off).
 */
#ifndef OFLOW_ORACLE_H
#define OFLOW_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- TV-L1 building blocks ---------------- */
int orc_gaussian_window(double sigma);
int orc_gaussian(float *I, int nx, int ny, double sigma);
float orc_bicubic_at(const float *in, float uu, float vv, int nx, int ny, int border_out);
void orc_bicubic_warp(const float *in, const float *u, const float *v, float *out, int nx,
                      int ny, int border_out);
void orc_zoom_size(int nx, int ny, int *nxx, int *nyy, float factor);
int orc_zoom_out(const float *I, float *Iout, int nx, int ny, float factor);
void orc_zoom_in(const float *I, float *Iout, int nx, int ny, int nxx, int nyy);
void orc_centered_gradient(const float *in, float *dx, float *dy, int nx, int ny);
void orc_divergence(const float *v1, const float *v2, float *div, int nx, int ny);
void orc_forward_gradient(const float *f, float *fx, float *fy, int nx, int ny);
void orc_normalize(float *I0, float *I1, int n);
int orc_tvl1_nscales(int w, int h, int nscales, float zfactor);

typedef struct {
    float tau, lambda, theta;
    int nscales;
    float zfactor;
    int warps;
    float epsilon;
    int max_iterations;
    /* 0: error summed left to right in float (the reference at one OpenMP
     *    thread); 1: summed in double and rounded once to float. */
    int error_mode;
} orc_tvl1_params;

/* Optional per-solve records.  iterations[s*warps + w] = inner iterations run
 * at scale s, warp w.  energy (if non-NULL) receives, per (s, w, n), the TV-L1
 * energy after the u update of iteration n, at index
 * (s*warps + w)*max_iterations + n (entries past the stop are untouched). */
typedef struct {
    int *iterations;
    double *energy;
} orc_tvl1_trace;

/* One pyramid level (tvl1.cpp:182-294). u1,u2 in/out; p (optional) 4*nx*ny. */
void orc_dual_tvl1(const float *I0, const float *I1, float *u1, float *u2, int nx, int ny,
                   const orc_tvl1_params *prm, float *p, int *iters, double *energy);

/* Full multiscale solve from float frames (tvl1.cpp:129-175). Returns the
 * number of scales used, or -1 on bad sizes.  trace may be NULL. */
int orc_tvl1(const float *I0, const float *I1, int w, int h, const orc_tvl1_params *prm,
             float *u, float *v, orc_tvl1_trace *trace);

/* TV-L1 energy of (u1,u2) at the linearisation (I1wx, I1wy, rho_c):
 * sum |grad u1| + |grad u2| (forward differences) + lambda * sum |rho|. */
double orc_tvl1_energy(const float *u1, const float *u2, const float *I1wx,
                       const float *I1wy, const float *rho_c, int nx, int ny, float lambda);

/* ---------------- Horn-Schunck ---------------- */
void orc_hs_downscale(const float *src, int w, int h, float *dst);
void orc_hs_warp(const float *src, const float *u, const float *v, int w, int h, float *out);
void orc_hs_derivatives(const float *I0, const float *I1w, int w, int h, float *Ix, float *Iy,
                        float *Iz);
void orc_hs_jacobi(const float *du0, const float *dv0, const float *Ix, const float *Iy,
                   const float *Iz, int w, int h, float alpha, float *du1, float *dv1);
void orc_upscale(const float *src, int w, int h, int nw, int nh, float scale, float *dst);
int orc_hs(const float *I0, const float *I1, int w, int h, float alpha, int nlevels,
           int nwarp, int nsolver, float *u, float *v);

/* ---------------- Lucas-Kanade ---------------- */
int orc_lk_filters(int spac_size, int temp_size, float *fs, float *ft);
/* Single step over a ring of T=temp_size u8 frames (frames[k] = slot k),
 * newest frame in slot iframe % T (lucaskanade.cu:54-71). */
int orc_lk(const uint8_t *const *frames, int nx, int ny, int spac_size, int temp_size,
           int window, int iframe, float *Vx, float *Vy);
/* Same on float frames I0 (older), I1 (newer), temporal filter of size 2. */
int orc_lk_f32(const float *I0, const float *I1, int nx, int ny, int spac_size, int window,
               float *Vx, float *Vy);
void orc_bilinear_warp(const float *src, const float *u, const float *v, int w, int h,
                       float *out);
int orc_pyrlk(const float *I0, const float *I1, int w, int h, int levels, int iters,
              int spac_size, int window, float *u, float *v);

/* ---------------- flow visualisation ---------------- */
/* flowToColor (src/tvl1/sequential/main.cpp:93-126): per pixel V = 8-bit
 * min(10|f|, 255), H = 8-bit (atan2(v,u) in degrees)/2 (negative angles
 * saturate to 0), S = 255, then HSV (H in 0..180) -> B, G, R bytes by the
 * hexcone formulas.  u, v planar w x h floats; bgr w*h*3 bytes. */
void orc_flow_to_color(const float *u, const float *v, int w, int h, uint8_t *bgr);

#ifdef __cplusplus
}
#endif

#endif
