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
// On the GPU this runs on the double-precision pipe (two conversions in, the
// IEEE double square root, one conversion out), which measured cheaper than
// a single-precision candidate with a residual test around the rounding
// midpoints.
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

// Hardware reciprocal estimate (PTX rcp.approx), refined below by one Newton
// step.  On the host the refined form is the plain correctly rounded
// reciprocal, which satisfies the same contract.
#ifdef __CUDA_ARCH__
__device__ __forceinline__ float rcp_est(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
#endif

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
