// Device checks of the approximation behind the exact fast forms of
// exact_math.cuh.  rcp_near_rn starts from the hardware's estimate
// instruction, whose rounding the host cannot reproduce, so its contract is
// checked on the device: exhaustively over its range of float bit patterns
// (which 1), and through the Markstein quotient on seeded pseudo-random
// operands (which 3).  oflow_selftest_math returns the number of operands that
// break the contract.
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"
#include "internal.hpp"

namespace oflow {
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// a float with a uniformly drawn exponent in [emin, emax], random mantissa and sign
__device__ __forceinline__ float draw(uint64_t h, int emin, int emax, bool sign) {
    const int e = emin + (int)((h >> 40) % (uint64_t)(emax - emin + 1));
    const uint32_t m = (uint32_t)h & 0x7fffffu;
    uint32_t bits = ((uint32_t)(e + 127) << 23) | m;
    if (sign && (h >> 63)) bits |= 0x80000000u;
    return __uint_as_float(bits);
}

__device__ __forceinline__ bool same_bits(float a, float b) {
    return __float_as_uint(a) == __float_as_uint(b) || (a != a && b != b);
}

__global__ void k_selftest(int which, uint32_t lo, uint32_t hi, uint64_t seed,
                           unsigned long long *count) {
    unsigned long long bad = 0;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi && i >= lo; i += stride) {
        if (which == 1) {  // rcp_near_rn is the correctly rounded reciprocal
            const float g = __uint_as_float(i);
            bad += !same_bits(rcp_near_rn(g), __frcp_rn(g));
        } else {  // Markstein quotient from rcp_near_rn equals IEEE division
            const uint64_t h = mix64(seed ^ ((uint64_t)i << 1)), h2 = mix64(h);
            const float g = (i & 1) ? draw(h, -40, 23, false) : 1.0f + draw(h, -20, 22, false);
            const float p = (i & 2) ? draw(h2, -99, 30, true) : draw(h2, -20, 20, true);
            if (rcp_in_range(g) && markstein_safe(p))
                bad += !same_bits(markstein(p, g, rcp_near_rn(g)), __fdiv_rn(p, g));
        }
    }
    for (int o = 16; o > 0; o >>= 1) bad += __shfl_down_sync(0xffffffffu, bad, o);
    if ((threadIdx.x & 31) == 0 && bad) atomicAdd(count, bad);
}

}  // namespace
}  // namespace oflow

extern "C" oflow_status oflow_selftest_math(int which, uint32_t lo, uint32_t hi,
                                            unsigned long long seed, unsigned long long *mismatches) {
    if (!mismatches || (which != 1 && which != 3) || hi < lo) return OFLOW_ERR_BAD_ARG;
    unsigned long long *d = nullptr;
    if (cudaMalloc(&d, sizeof(*d)) != cudaSuccess) {
        cudaGetLastError();
        return OFLOW_ERR_CUDA;
    }
    cudaError_t e = cudaMemset(d, 0, sizeof(*d));
    if (e == cudaSuccess) {
        oflow::k_selftest<<<oflow::kNumSMs * 8, 256>>>(which, lo, hi, seed, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(mismatches, d, sizeof(*d), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return OFLOW_ERR_CUDA;
    }
    return OFLOW_OK;
}
