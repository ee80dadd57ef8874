// Flow visualisation: the demos' flowToColor (src/tvl1/sequential/main.cpp:
// 93-126) as one kernel writing B, G, R bytes into a device buffer (no window).
//
// Per pixel: V = 8-bit min(10 |f|, 255); H = 8-bit atan2(v, u) in degrees / 2,
// negative angles saturating to 0 as the reference's float -> CV_8U
// conversion does; S = 255; then HSV -> BGR by the hexcone model with H in
// 0..180 and S, V in 0..255 (the scaling of the reference's cvtColor call).
// Every step is single precision with one rounding per operation (the library
// is built without contraction); the angle is atan2 correctly rounded to
// float (a float fast path decides wherever it provably agrees, double
// precision elsewhere).  8-bit conversions round to nearest even and saturate.
//
// One thread converts 4 consecutive pixels of a row: two float4 loads, three
// 32-bit stores when the row allows it, bytes otherwise.  8 B in and 3 B out
// per pixel: an HBM-bound kernel.
#include <cuda_runtime.h>
#include <stdint.h>

#include "color.hpp"
#include "common.cuh"
#include "internal.hpp"

namespace oflow {

namespace {

constexpr int kColorNT = 128;

// Rounding to an integer without the conversion pipe: for |x| < 2^22,
// x + 1.5*2^23 rounds x to an integer (nearest even, as rintf), whose value
// sits in the low mantissa bits.  Returns that integer and sets r = rintf(x).
constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23
constexpr int kMagicBits = 0x4B400000;
__device__ __forceinline__ int rint_small(float x, float &r) {
    const float t = x + kMagic;
    r = t - kMagic;
    return __float_as_int(t) - kMagicBits;
}
// floorf(x) for 0 <= |x| < 2^22, as a float and an integer
__device__ __forceinline__ int floor_small(float x, float &fl) {
    float r;
    const int k = rint_small(x, r);
    const bool over = r > x;
    fl = over ? r - 1.0f : r;
    return over ? k - 1 : k;
}

// B | G << 8 | R << 16 of one flow vector.  Every byte is the 8-bit saturating
// round-to-nearest-even conversion of the reference; the operands are known to
// lie in [0, 255] (V after its clamp, the colour channels) or in [-91, 91]
// (the hue), so rint_small replaces rintf and the float<->int conversions.
__device__ __forceinline__ uint32_t flow_bgr(float fu, float fv) {
    const float hue_scale = (float)(180.0 / 3.14159265358979323846 / 2.0);
    const float mag = sqrtf(fu * fu + fv * fv);
    float m = mag * 10.0f;
    if (m > 255.0f) m = 255.0f;
    float vr;  // the V byte as a float
    rint_small(m, vr);
    if (!(m == m)) vr = 0.0f;  // NaN converts to 0
    // hue byte = rint(RN(RN(atan2) * scale)) with atan2 correctly rounded to
    // float.  atan2f is within 3 ulp (CUDA's documented bound), which moves
    // the scaled angle (|.| <= 90) by less than 3.5e-5 including the product's
    // rounding; only when that lies within 1e-4 of a rounding boundary k + 1/2
    // can the byte differ, and then the double-precision atan2 decides.
    float hf = atan2f(fv, fu) * hue_scale;
    float fl;
    floor_small(hf, fl);
    if (fabsf(hf - (fl + 0.5f)) < 1e-4f || !(fabsf(hf) <= 91.0f))
        hf = (float)atan2((double)fv, (double)fu) * hue_scale;
    float hr;  // the H byte as a float
    if (rint_small(hf, hr) < 0 || !(hf == hf)) hr = 0.0f;  // negative angles and NaN saturate to 0
    const float hh = hr * (6.0f / 180.0f);
    float sf;
    int sector = floor_small(hh, sf);
    float f = hh - sf;
    if (sector < 0 || sector > 5) {
        sector = 0;
        f = 0.0f;
    }
    const float s = 255.0f * (1.0f / 255.0f);
    const float vv = vr * (1.0f / 255.0f);
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
    float unused;
    const uint32_t B8 = (uint32_t)rint_small(b * 255.0f, unused);
    const uint32_t G8 = (uint32_t)rint_small(g * 255.0f, unused);
    const uint32_t R8 = (uint32_t)rint_small(r * 255.0f, unused);
    return B8 | (G8 << 8) | (R8 << 16);
}

__global__ void __launch_bounds__(kColorNT) k_flow_to_color(ColorJobs jobs) {
    const ColorJob jb = jobs.j[blockIdx.z];
    const int y = blockIdx.y;
    const int x0 = (blockIdx.x * kColorNT + threadIdx.x) * 4;
    if (x0 >= jobs.w) return;
    const float *ur = jb.u + (size_t)y * jb.fpitch;
    const float *vr = jb.v + (size_t)y * jb.fpitch;
    uint8_t *o = jb.bgr + (size_t)y * jb.bpitch + (size_t)x0 * 3;
    if (jb.vec && x0 + 3 < jobs.w) {
        const float4 a = *reinterpret_cast<const float4 *>(ur + x0);
        const float4 b = *reinterpret_cast<const float4 *>(vr + x0);
        const uint32_t c0 = flow_bgr(a.x, b.x), c1 = flow_bgr(a.y, b.y);
        const uint32_t c2 = flow_bgr(a.z, b.z), c3 = flow_bgr(a.w, b.w);
        uint32_t *o32 = reinterpret_cast<uint32_t *>(o);
        o32[0] = c0 | (c1 << 24);
        o32[1] = (c1 >> 8) | (c2 << 16);
        o32[2] = (c2 >> 16) | (c3 << 8);
        return;
    }
    for (int k = 0; k < 4 && x0 + k < jobs.w; k++) {
        const uint32_t c = flow_bgr(ur[x0 + k], vr[x0 + k]);
        o[3 * k + 0] = (uint8_t)c;
        o[3 * k + 1] = (uint8_t)(c >> 8);
        o[3 * k + 2] = (uint8_t)(c >> 16);
    }
}

}  // namespace

void launch_flow_to_color(ColorJobs &jobs, int n, cudaStream_t st) {
    for (int i = 0; i < n; i++) {
        const ColorJob &j = jobs.j[i];
        // float4 loads and 32-bit stores need 16-byte rows of u, v and 4-byte rows of bgr
        jobs.j[i].vec = ((reinterpret_cast<uintptr_t>(j.u) | reinterpret_cast<uintptr_t>(j.v)) & 15u) == 0 &&
                        (j.fpitch % 4) == 0 && (reinterpret_cast<uintptr_t>(j.bgr) & 3u) == 0 &&
                        (j.bpitch % 4) == 0;
    }
    dim3 g(div_up(jobs.w, 4 * kColorNT), jobs.h, n);
    k_flow_to_color<<<g, kColorNT, 0, st>>>(jobs);
}

}  // namespace oflow
