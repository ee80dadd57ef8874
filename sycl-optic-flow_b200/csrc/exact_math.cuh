// Exactly rounded single-precision helpers shared by host and device code.
// Each function returns bit-for-bit what the reference's x86 build computes
// for the same expression (IEEE single/double, no contraction), but with
// cheaper instruction sequences on the GPU.  They are compiled on the host as
// well, so tests can check them against the plain expressions on the CPU.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

namespace oflow {

#ifdef __CUDA_ARCH__
__device__ __forceinline__ float __int_as_float_hd(int i) { return __int_as_float(i); }
__device__ __forceinline__ int __float_as_int_hd(float f) { return __float_as_int(f); }
#else
inline float __int_as_float_hd(int i) { float f; memcpy(&f, &i, 4); return f; }
inline int __float_as_int_hd(float f) { int i; memcpy(&i, &f, 4); return i; }
#endif

// Single-precision hypot exactly as glibc's hypotf: the squares are exact in
// double, one rounding for the sum, one for the square root, one to single.
__host__ __device__ __forceinline__ float hypot_ref(float a, float b) {
    const double da = a, db = b;
    return (float)sqrt(da * da + db * db);
}

#ifdef __CUDA_ARCH__
#define OF_FMAF(a, b, c) __fmaf_rn(a, b, c)
#define OF_RCP(x) __frcp_rn(x)
#else
#define OF_FMAF(a, b, c) fmaf(a, b, c)
#define OF_RCP(x) (1.0f / (x))
#endif

// Hardware estimates (PTX rsqrt.approx / rcp.approx), refined below by one
// Newton step each.  On the host the refined forms are the plain correctly
// rounded operations, which satisfy the same contracts.
#ifdef __CUDA_ARCH__
__device__ __forceinline__ float rsqrt_est(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float rcp_est(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
#endif

// sqrt(x) within one ulp (not necessarily correctly rounded) for positive
// normal x: y = x*r from the reciprocal square-root estimate r, then one
// Newton step y + (r/2)(x - y^2).  The device tests check every positive
// normal float against the correctly rounded sqrtf.
__host__ __device__ __forceinline__ float sqrt_near(float x) {
#ifdef __CUDA_ARCH__
    const float r = rsqrt_est(x);
    const float y = x * r;
    const float e = __fmaf_rn(-y, y, x);
    return __fmaf_rn(0.5f * r, e, y);
#else
    return sqrtf(x);
#endif
}

// RN(1/g) for g in [kRcpLo, kRcpHi): the reciprocal estimate r, then one
// Newton step r + r(1 - g r) with the residual formed exactly by a fused
// multiply-add.  The device tests check every float of the range against the
// correctly rounded reciprocal; rcp_in_range says whether g lies in it.
constexpr float kRcpLo = 0x1p-40f, kRcpHi = 0x1p24f;
__host__ __device__ __forceinline__ bool rcp_in_range(float g) { return g >= kRcpLo && g < kRcpHi; }
__host__ __device__ __forceinline__ float rcp_near_rn(float g) {
#ifdef __CUDA_ARCH__
    const float r = rcp_est(g);
    const float e = __fmaf_rn(-g, r, 1.0f);
    return __fmaf_rn(r, e, r);
#else
    return 1.0f / g;
#endif
}

// hypot_ref without double arithmetic on the common path.  With S = a^2+b^2
// held exactly as float pairs, y0 = sqrt_near(RN(bh+sh)) is within 1.5 ulp of
// sqrt(S) (one ulp from sqrt_near, half an ulp from rounding the sum), so the
// correctly rounded result is y0 or one of its neighbours.  The residual
// e = S - y0^2 (error < 2^-46 S) places sqrt(S) relative to the midpoints
// y0 +- ulp/2 (at |e| = y0*ulp to first order, the second-order term far
// below the margin even with y0 an ulp off).  When it is
// more than 2^-20 of that distance away, single rounding of sqrt(S) and the
// reference's double-then-single rounding agree, and the fast answer is
// certain; otherwise (and for tiny, huge or non-finite input) the double
// formula decides.  The lower bound 2^-50 on the larger operand keeps every
// low-order product term (bl, yl) a normal number, so the rounding errors of
// the subnormal small-operand terms stay far below the 2^-20 margin.
// hypot_try returns the fast candidate and whether it is certain, without
// branches, so two lanes can share one branch to the fallback.
__host__ __device__ __forceinline__ float hypot_try(float a, float b, bool &ok) {
    a = fabsf(a);
    b = fabsf(b);
    const float big = fmaxf(a, b), small = fminf(a, b);
    const float bh = big * big, bl = OF_FMAF(big, big, -bh);
    const float sh = small * small, sl = OF_FMAF(small, small, -sh);
    const float y0 = sqrt_near(bh + sh);
    const float yh = y0 * y0, yl = OF_FMAF(y0, y0, -yh);
    // (bh - yh) and the following add are exact (Sterbenz); the low parts
    // carry errors far below the threshold
    const float e = ((bh - yh) + sh) + ((bl + sl) - yl);
    const float ulp = __int_as_float_hd((__float_as_int_hd(y0) & 0x7f800000) - (23 << 23));
    const float T = y0 * ulp;
    const float margin = T * 0x1p-20f;
    const bool up = e > T + margin, dn = e < -(T + margin), mid = fabsf(e) < T - margin;
    // fmaxf / fminf drop a NaN operand; the sum keeps it (and big <= s <= 2 big)
    const float s = a + b;
    const bool in_range = s >= 0x1p-49f && s < 0x1p60f;
    const bool zero = small == 0.0f && s == s;  // sqrt(x^2) = |x| exactly
    ok = (in_range && (up || dn || mid)) || zero;
    const float y = __int_as_float_hd(__float_as_int_hd(y0) + (up ? 1 : 0) - (dn ? 1 : 0));
    return zero ? big : y;
}

__host__ __device__ __forceinline__ float hypot_fast(float a, float b) {
    bool ok;
    const float y = hypot_try(a, b, ok);
    return ok ? y : hypot_ref(a, b);
}

// Both hypots of a dual update with one (rarely taken) branch to the fallback.
__host__ __device__ __forceinline__ void hypot2_fast(float a1, float b1, float a2, float b2,
                                                     float &h1, float &h2) {
    bool ok1, ok2;
    h1 = hypot_try(a1, b1, ok1);
    h2 = hypot_try(a2, b2, ok2);
    if (!(ok1 && ok2)) {
        if (!ok1) h1 = hypot_ref(a1, b1);
        if (!ok2) h2 = hypot_ref(a2, b2);
    }
}

// p / g correctly rounded (IEEE division) from y = RN(1/g): q0 = RN(p*y),
// r = p - q0*g (exact by FMA), q = RN(q0 + r*y) (Markstein).  Valid while
// neither the quotient nor p underflows: |p| > 2^-100 with g < 2^24 keeps the
// quotient above 2^-124; and for p = +0.  markstein_safe says so for p; other
// p take the plain division.
__host__ __device__ __forceinline__ float markstein(float p, float g, float y) {
    const float q0 = p * y;
    const float r = OF_FMAF(-q0, g, p);
    return OF_FMAF(r, y, q0);
}

__host__ __device__ __forceinline__ bool markstein_safe(float p) {
    return fabsf(p) > 0x1p-100f || __float_as_int_hd(p) == 0;
}

__host__ __device__ __forceinline__ float div_by_rcp(float p, float g, float y) {
    if (markstein_safe(p)) return markstein(p, g, y);
    return p / g;
}

}  // namespace oflow
