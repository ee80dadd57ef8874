// TEST INFRASTRUCTURE ONLY.  C entry points around the reference's own
// Horn-Schunck and Lucas-Kanade CUDA kernels, compiled where they lie in the
// reference checkout (src/hs/cuda/kernels/*.cuh are included below;
// src/lk/cuda/{lucaskanade,kernels/kernels}.cu are compiled as their own
// translation units by build_ref.sh).  Nothing here is part of the product:
// the tests use it to check the library's HS/LK kernels and the oracle's
// restatement against the reference's kernels on identical inputs.
//
// Only the kernels whose every access stays in bounds for the inputs these
// entry points accept are run:
//   JacobiIteration<32,6>   solverKernel.cuh:41-153   (through SolveForUpdate)
//   AddKernel               addKernel.cuh:28-36        (through Add)
//   DownscaleKernel         downscaleKernel.cuh:27-40  (through Downscale)
//   temp_convolution_GPU, spac_convolution2D_x_GPU, luca_kanade_1step_GPU
//                           src/lk/cuda/kernels/kernels.cu:14-30, 44-80, 134-181
//   spac_convolution2D_y_GPU kernels.cu:83-121, only for square frames: its
//                           bottom-border test compares the row with the width
//                           (:106), which is in bounds and correct when nx == ny
//                           and reads past the frame when ny < nx.
// WarpingKernel, ComputeDerivativesKernel and UpscaleKernel are never run:
// each reads outside its buffers (warpingKernel.cuh:38-40,
// derivativesKernel.cuh:39, upscaleKernel.cuh:33-39).
//
// All entry points take and return host arrays, allocate and free their own
// device buffers, synchronise, and return 0 on success, -1 on a bad argument,
// -2 on a CUDA error.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <iostream>
#include <vector>

// The reference HS kernels and their host wrappers (static functions in the
// headers, so they are compiled into this translation unit).
#include "kernels/solverKernel.cuh"
#include "kernels/addKernel.cuh"
#include "kernels/downscaleKernel.cuh"

// The reference LucasKanade class.  Its filter taps and derivative planes are
// private members; the harness reads them, so `private` is widened for this
// one include.  lucaskanade.cu itself is compiled unmodified in its own
// translation unit; the class layout does not depend on access specifiers.
#define private public
#include "lucaskanade.cuh"
#undef private

namespace {

struct Dev {
    void *p = nullptr;
    ~Dev() {
        if (p) cudaFree(p);
    }
    bool alloc(size_t bytes) { return cudaMalloc(&p, bytes) == cudaSuccess; }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

int finish() {
    if (cudaDeviceSynchronize() != cudaSuccess) return -2;
    if (cudaGetLastError() != cudaSuccess) return -2;
    return 0;
}

// Copy a w x h host plane into a device plane of row stride s (floats).
bool put_strided(float *d, const float *h, int w, int hgt, int s) {
    return cudaMemcpy2D(d, sizeof(float) * s, h, sizeof(float) * w, sizeof(float) * w, hgt,
                        cudaMemcpyHostToDevice) == cudaSuccess;
}
bool get_strided(float *h, const float *d, int w, int hgt, int s) {
    return cudaMemcpy2D(h, sizeof(float) * w, d, sizeof(float) * s, sizeof(float) * w, hgt,
                        cudaMemcpyDeviceToHost) == cudaSuccess;
}

}  // namespace

extern "C" {

int refg_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

// 2x2 box downscale of a w x h plane by the reference's Downscale /
// DownscaleKernel.  The kernel indexes its source with the stride it is given
// for the destination (downscaleKernel.cuh:36-39; flow.cu:138-142 passes the
// new level's stride), so the harness gives it the source width as that stride
// and a destination of the same row stride: every source read is then the
// intended pixel.  The kernel writes output columns < w/2-1 and rows < h/2-1
// (:32); dst (w/2 x h/2) keeps its given values in the last column and row.
int refg_hs_downscale(const float *src, int w, int h, float *dst) {
    if (!src || !dst || w < 4 || h < 4) return -1;
    const int nw = w / 2, nh = h / 2;
    Dev ds, dd;
    if (!ds.alloc(sizeof(float) * w * h) || !dd.alloc(sizeof(float) * w * nh)) return -2;
    if (cudaMemcpy(ds.p, src, sizeof(float) * w * h, cudaMemcpyHostToDevice) != cudaSuccess)
        return -2;
    if (!put_strided(dd.as<float>(), dst, nw, nh, w)) return -2;
    Downscale(ds.as<float>(), w, h, w, nw, nh, w, dd.as<float>());
    if (finish()) return -2;
    return get_strided(dst, dd.as<float>(), nw, nh, w) ? 0 : -2;
}

// nsweeps Jacobi sweeps from du = dv = 0, by the reference's SolveForUpdate
// (JacobiIteration<32,6>) with the buffer swap of flow.cu:186-193.  Planes
// are w x h on the host and `stride` floats per row on the device.
int refg_hs_jacobi(const float *Ix, const float *Iy, const float *Iz, int w, int h, int stride,
                   float alpha, int nsweeps, float *du, float *dv) {
    if (!Ix || !Iy || !Iz || !du || !dv || w < 1 || h < 1 || stride < w || nsweeps < 0)
        return -1;
    const size_t bytes = sizeof(float) * (size_t)stride * h;
    Dev dIx, dIy, dIz, a0, b0, a1, b1;
    if (!dIx.alloc(bytes) || !dIy.alloc(bytes) || !dIz.alloc(bytes) || !a0.alloc(bytes) ||
        !b0.alloc(bytes) || !a1.alloc(bytes) || !b1.alloc(bytes))
        return -2;
    for (Dev *d : {&dIx, &dIy, &dIz, &a0, &b0, &a1, &b1})
        if (cudaMemset(d->p, 0, bytes) != cudaSuccess) return -2;
    if (!put_strided(dIx.as<float>(), Ix, w, h, stride) ||
        !put_strided(dIy.as<float>(), Iy, w, h, stride) ||
        !put_strided(dIz.as<float>(), Iz, w, h, stride))
        return -2;
    float *du0 = a0.as<float>(), *dv0 = b0.as<float>();
    float *du1 = a1.as<float>(), *dv1 = b1.as<float>();
    for (int it = 0; it < nsweeps; ++it) {
        SolveForUpdate(du0, dv0, dIx.as<float>(), dIy.as<float>(), dIz.as<float>(), w, h, stride,
                       alpha, du1, dv1);
        Swap(du0, du1);
        Swap(dv0, dv1);
    }
    if (finish()) return -2;
    return get_strided(du, du0, w, h, stride) && get_strided(dv, dv0, w, h, stride) ? 0 : -2;
}

// out = a + b over n floats by the reference's Add (AddKernel).
int refg_hs_add(const float *a, const float *b, int n, float *out) {
    if (!a || !b || !out || n < 1) return -1;
    Dev da, db, dc;
    const size_t bytes = sizeof(float) * (size_t)n;
    if (!da.alloc(bytes) || !db.alloc(bytes) || !dc.alloc(bytes)) return -2;
    if (cudaMemcpy(da.p, a, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(db.p, b, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return -2;
    Add(da.as<float>(), db.as<float>(), n, dc.as<float>());
    if (finish()) return -2;
    return cudaMemcpy(out, dc.p, bytes, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -2;
}

// The FIR taps of a LucasKanade object (getfilters, lucaskanade.cu:79-161).
// Sizes the reference has no table for are rejected (it prints and leaves the
// taps unset).
int refg_lk_filters(int spac, int temp, float *fx, float *fy, float *ft) {
    const bool s_ok = spac == 1 || spac == 3 || spac == 5 || spac == 7 || spac == 9;
    const bool t_ok = temp == 1 || temp == 2 || temp == 3 || temp == 5 || temp == 7 || temp == 9;
    if (!fx || !fy || !ft || !s_ok || !t_ok) return -1;
    LucasKanade lk(spac, temp, 3, 8, 8);
    std::memcpy(fx, lk.filt_x, sizeof(float) * spac);
    std::memcpy(fy, lk.filt_y, sizeof(float) * spac);
    std::memcpy(ft, lk.filt_t, sizeof(float) * temp);
    return finish();
}

// One reference LucasKanade::lucas_kanade call on a ring of `temp` frames
// (slot k holds ring[k*nx*ny ...], loaded with copy_frames_circularbuffer_GPU_wrapper
// as frame number k).  Square frames only (see the header comment).  Vx, Vy:
// the flow (pixels within the window radius of the border are whatever the
// reference left there: it never writes them); Ix, Iy, It: its derivative
// planes (any may be NULL).
int refg_lk_class(const uint8_t *ring, int nx, int ny, int spac, int temp, int window, int iframe,
                  float *Vx, float *Vy, float *Ix, float *Iy, float *It) {
    if (!ring || !Vx || !Vy || nx != ny || nx < 16 || window < 1 || window % 2 == 0 ||
        iframe < 0)
        return -1;
    float tmp[9];
    if (refg_lk_filters(spac, temp, tmp, tmp, tmp)) return -1;
    const int n = nx * ny;
    LucasKanade lk(spac, temp, window, nx, ny);
    std::vector<unsigned char> frame(n);
    for (int k = 0; k < temp; ++k) {
        std::memcpy(frame.data(), ring + (size_t)k * n, n);
        lk.copy_frames_circularbuffer_GPU_wrapper(frame.data(), temp, k, n);
    }
    lk.lucas_kanade(Vx, Vy, iframe);
    if (finish()) return -1;
    const size_t b = sizeof(float) * n;
    if (Ix && cudaMemcpy(Ix, lk.d_Ix, b, cudaMemcpyDeviceToHost) != cudaSuccess) return -2;
    if (Iy && cudaMemcpy(Iy, lk.d_Iy, b, cudaMemcpyDeviceToHost) != cudaSuccess) return -2;
    if (It && cudaMemcpy(It, lk.d_It, b, cudaMemcpyDeviceToHost) != cudaSuccess) return -2;
    return 0;
}

// The same computation for frames of any shape, from the reference's kernel
// wrappers: It by temp_convolution_GPU_wrapper, Ix by
// spac_convolution2D_x_GPU_wrapper on the oldest ring frame
// (lucaskanade.cu:54-62), Iy by the same x-filter applied to the transposed
// frame and transposed back (the y-filter with its bottom border taken at the
// height), then luca_kanade_1step_GPU_wrapper.  The flow planes start at zero,
// so pixels within the window radius of the border read 0.
int refg_lk_parts(const uint8_t *ring, int nx, int ny, int spac, int temp, int window, int iframe,
                  float *Vx, float *Vy, float *Ix, float *Iy, float *It) {
    if (!ring || !Vx || !Vy || nx < 16 || ny < 16 || window < 1 || window % 2 == 0 || iframe < 0)
        return -1;
    float fx[9], fy[9], ft[9];
    if (refg_lk_filters(spac, temp, fx, fy, ft)) return -1;
    const int n = nx * ny;
    const size_t fb = sizeof(float) * n;
    Dev dring, dT, dfx, dft, dIx, dIy, dIyT, dIt, dVx, dVy;
    if (!dring.alloc((size_t)temp * n) || !dT.alloc(n) || !dfx.alloc(sizeof(float) * spac) ||
        !dft.alloc(sizeof(float) * temp) || !dIx.alloc(fb) || !dIy.alloc(fb) ||
        !dIyT.alloc(fb) || !dIt.alloc(fb) || !dVx.alloc(fb) || !dVy.alloc(fb))
        return -2;
    if (cudaMemcpy(dring.p, ring, (size_t)temp * n, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dfx.p, fx, sizeof(float) * spac, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dft.p, ft, sizeof(float) * temp, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(dVx.p, 0, fb) != cudaSuccess || cudaMemset(dVy.p, 0, fb) != cudaSuccess)
        return -2;
    const int oldest = (iframe + 1) % temp;
    const uint8_t *f = ring + (size_t)oldest * n;
    std::vector<uint8_t> ft_host(n);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) ft_host[(size_t)x * ny + y] = f[(size_t)y * nx + x];
    if (cudaMemcpy(dT.p, ft_host.data(), n, cudaMemcpyHostToDevice) != cudaSuccess) return -2;
    unsigned char *d_oldest = dring.as<unsigned char>() + (size_t)oldest * n;
    temp_convolution_GPU_wrapper(iframe, dIt.as<float>(), dring.as<unsigned char>(), nx, ny,
                                 dft.as<float>(), temp);
    spac_convolution2D_x_GPU_wrapper(dIx.as<float>(), d_oldest, nx, ny, dfx.as<float>(), spac);
    spac_convolution2D_x_GPU_wrapper(dIyT.as<float>(), dT.as<unsigned char>(), ny, nx,
                                     dfx.as<float>(), spac);
    if (finish()) return -2;
    std::vector<float> yt(n), yy(n);
    if (cudaMemcpy(yt.data(), dIyT.p, fb, cudaMemcpyDeviceToHost) != cudaSuccess) return -2;
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) yy[(size_t)y * nx + x] = yt[(size_t)x * ny + y];
    if (cudaMemcpy(dIy.p, yy.data(), fb, cudaMemcpyHostToDevice) != cudaSuccess) return -2;
    luca_kanade_1step_GPU_wrapper(Vx, Vy, dVx.as<float>(), dVy.as<float>(), dIx.as<float>(),
                                  dIy.as<float>(), dIt.as<float>(), spac, temp, window, nx, ny);
    if (finish()) return -2;
    if (Ix && cudaMemcpy(Ix, dIx.p, fb, cudaMemcpyDeviceToHost) != cudaSuccess) return -2;
    if (Iy) std::memcpy(Iy, yy.data(), fb);
    if (It && cudaMemcpy(It, dIt.p, fb, cudaMemcpyDeviceToHost) != cudaSuccess) return -2;
    return 0;
}

}  // extern "C"
