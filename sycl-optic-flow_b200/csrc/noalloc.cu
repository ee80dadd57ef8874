// Horn-Schunck for callers that cannot allocate device memory.
//
// Some callers of this library must not call cudaMalloc: real-time frame
// loops that cannot take the device-wide synchronisation a cudaMalloc/cudaFree
// may imply, and hosts that hand the library a fixed memory budget up front.
// oflow_hs_noalloc serves them: its scratch is one static device array,
// allocated when the library's device code is loaded and held by every GPU
// that loads it until the process exits.
#include <cuda_runtime.h>

#include <mutex>

#include "hs.hpp"
#include "internal.hpp"

namespace {

// Capacity of the static scratch: 8 MiB.  With one level a frame needs 64 B
// per pixel (320x240: 4.9 MB), so frames up to about 131,000 pixels fit; more
// levels add up to 8/3 B per pixel (the pyramid).
constexpr size_t kStaticScratchBytes = size_t(8) << 20;
__device__ __align__(256) unsigned char g_hs_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch_addr[kMaxDevices] = {};

// Device address of g_hs_scratch on the current device.  In host code the
// array's name is only a host-side stand-in, so the address is looked up once
// per device with that device current and cached for the process (a device
// reset, after which the array may sit elsewhere, is not followed).
cudaError_t scratch_address(void **out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_hs_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" oflow_status oflow_hs_noalloc(const float *I0, const float *I1, int width, int height,
                                         int pitch, const oflow_hs_params *p, float *u, float *v,
                                         int out_pitch, void *stream) {
    if (!I0 || !I1 || !u || !v || !p || width < 1 || height < 1) return OFLOW_ERR_BAD_ARG;
    if ((pitch && pitch < width) || (out_pitch && out_pitch < width)) return OFLOW_ERR_BAD_ARG;
    if (p->nlevels < 1 || p->nlevels > 16 || p->nwarp < 0 || p->nsolver < 0)
        return OFLOW_ERR_BAD_ARG;
    const size_t need = oflow::hs_scratch_bytes(width, height, p->nlevels);
    if (need == 0) return OFLOW_ERR_BAD_ARG;            // levels below 1x1
    if (need > kStaticScratchBytes) return OFLOW_ERR_BAD_ARG;  // beyond the static capacity
    void *scratch = nullptr;
    if (scratch_address(&scratch) != cudaSuccess) {
        cudaGetLastError();
        return OFLOW_ERR_CUDA;
    }
    try {
        oflow::hs_enqueue_into(scratch, I0, I1, width, height, pitch, *p, u, v, out_pitch,
                               static_cast<cudaStream_t>(stream));
    } catch (const oflow::Error &e) {
        return e.code;
    } catch (...) {
        return OFLOW_ERR_CUDA;
    }
    return OFLOW_OK;
}
