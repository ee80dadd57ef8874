/*
 * Minimal stand-in for the six MKL BLAS-1 routines that the reference's
 * sequential TV-L1 calls (src/tvl1/sequential/tvl1.cpp:213-214, :322-325,
 * :353-356; src/tvl1/sequential/mask/mask.cpp:242-244).  MKL is not part of
 * this toolchain, so the reference is compiled against these plain loops.
 *
 * Semantics follow the BLAS reference definitions:
 *   sscal  x := a*x                   saxpy  y := a*x + y (one multiply, one add)
 *   isamax first index of max |x_i|   isamin first index of min |x_i| (0-based,
 *                                     as MKL's CBLAS interface returns them)
 *   dasum  sum |x_i|, left to right   dscal  x := a*x
 *
 * This file is test infrastructure: it is only compiled into oracle/_ref.
 */
#ifndef ORACLE_REF_SHIM_MKL_H
#define ORACLE_REF_SHIM_MKL_H

#include <cmath>
#include <cstddef>

typedef long long MKL_INT;

static inline void cblas_sscal(MKL_INT n, float a, float *x, MKL_INT incx) {
    for (MKL_INT i = 0; i < n; i++) x[i * incx] = a * x[i * incx];
}

static inline void cblas_dscal(MKL_INT n, double a, double *x, MKL_INT incx) {
    for (MKL_INT i = 0; i < n; i++) x[i * incx] = a * x[i * incx];
}

static inline void cblas_saxpy(MKL_INT n, float a, const float *x, MKL_INT incx,
                               float *y, MKL_INT incy) {
    for (MKL_INT i = 0; i < n; i++) {
        const float ax = a * x[i * incx];
        y[i * incy] = ax + y[i * incy];
    }
}

static inline std::size_t cblas_isamax(MKL_INT n, const float *x, MKL_INT incx) {
    std::size_t best = 0;
    float bv = -1.0f;
    for (MKL_INT i = 0; i < n; i++) {
        const float a = std::fabs(x[i * incx]);
        if (a > bv) { bv = a; best = (std::size_t)i; }
    }
    return best;
}

static inline std::size_t cblas_isamin(MKL_INT n, const float *x, MKL_INT incx) {
    std::size_t best = 0;
    float bv = INFINITY;
    for (MKL_INT i = 0; i < n; i++) {
        const float a = std::fabs(x[i * incx]);
        if (a < bv) { bv = a; best = (std::size_t)i; }
    }
    return best;
}

static inline double cblas_dasum(MKL_INT n, const double *x, MKL_INT incx) {
    double s = 0.0;
    for (MKL_INT i = 0; i < n; i++) s += std::fabs(x[i * incx]);
    return s;
}

#endif
