// Flow visualisation (flowToColor) into B, G, R bytes on the device.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace oflow {

struct ColorJob {
    const float *u, *v;  // device planes
    int fpitch;          // floats per row of u and v
    uint8_t *bgr;        // device, 3 bytes per pixel
    int bpitch;          // bytes per row of bgr
    int vec;             // set by the launcher: aligned fast path allowed
};

constexpr int kColorMaxJobs = 32;  // per launch (kernel parameter space)

struct ColorJobs {
    ColorJob j[kColorMaxJobs];
    int w, h;
};

// Converts jobs.j[0..n) (all w x h); n <= kColorMaxJobs.
void launch_flow_to_color(ColorJobs &jobs, int n, cudaStream_t st);

}  // namespace oflow
