// Host-side internals shared by the solver plans and the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "oflow.h"

namespace oflow {

// Error carried to the C ABI boundary and turned into a status code there.
struct Error : std::runtime_error {
    oflow_status code;
    Error(oflow_status c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define OF_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            throw ::oflow::Error(e_ == cudaErrorMemoryAllocation ? OFLOW_ERR_OOM          \
                                                                 : OFLOW_ERR_CUDA,        \
                                 std::string(#call) + ": " + cudaGetErrorString(e_));      \
    } while (0)

#define OF_CHECK(cond, msg)                                                                \
    do {                                                                                   \
        if (!(cond)) throw ::oflow::Error(OFLOW_ERR_BAD_ARG, msg);                         \
    } while (0)

// Owned device allocation.
class DevBuf {
  public:
    DevBuf() = default;
    explicit DevBuf(size_t bytes) { alloc(bytes); }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    void alloc(size_t bytes) {
        release();
        if (bytes) OF_CUDA(cudaMalloc(&p_, bytes));
        n_ = bytes;
    }
    void release() {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        n_ = 0;
    }
    template <typename T> T *as() const { return static_cast<T *>(p_); }
    size_t bytes() const { return n_; }

  private:
    void *p_ = nullptr;
    size_t n_ = 0;
};

// Carves typed sub-buffers out of one allocation (256-byte aligned).
class Arena {
  public:
    size_t reserve(size_t bytes) {
        const size_t off = (size_ + 255) & ~size_t(255);
        size_ = off + bytes;
        return off;
    }
    void commit() { buf_.alloc(size_); }
    template <typename T> T *at(size_t off) const {
        return reinterpret_cast<T *>(buf_.as<char>() + off);
    }
    size_t size() const { return size_; }

  private:
    size_t size_ = 0;
    DevBuf buf_;
};

// An int in pinned host memory that kernels can set through its device
// address: an error flag the host reads without synchronising.
class HostFlag {
  public:
    HostFlag() {
        OF_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&h_), sizeof(int), cudaHostAllocMapped));
        *h_ = 0;
        OF_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void **>(&d_), h_, 0));
    }
    ~HostFlag() {
        if (h_) cudaFreeHost(h_);
    }
    HostFlag(const HostFlag &) = delete;
    HostFlag &operator=(const HostFlag &) = delete;
    int *device() const { return d_; }
    // sets the flag from the host, as a kernel would (failure injection)
    void raise() { *reinterpret_cast<volatile int *>(h_) = 1; }
    // the flag's value, cleared
    int take() {
        const int v = *reinterpret_cast<volatile int *>(h_);
        if (v) *reinterpret_cast<volatile int *>(h_) = 0;
        return v;
    }

  private:
    int *h_ = nullptr, *d_ = nullptr;
};

// A captured launch sequence replayed as one CUDA graph.
class Graph {
  public:
    ~Graph() { reset(); }
    void reset() {
        if (exec_) cudaGraphExecDestroy(exec_);
        if (graph_) cudaGraphDestroy(graph_);
        exec_ = nullptr;
        graph_ = nullptr;
    }
    bool ready() const { return exec_ != nullptr; }
    template <typename F> void capture(cudaStream_t s, F &&record) {
        reset();
        OF_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        try {
            record(s);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(s, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        OF_CUDA(cudaStreamEndCapture(s, &graph_));
        OF_CUDA(cudaGraphInstantiate(&exec_, graph_, 0));
    }
    void launch(cudaStream_t s) { OF_CUDA(cudaGraphLaunch(exec_, s)); }

  private:
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
};

// Copies a 2-D image (host or device, any pitch) into a dense device plane.
void stage_image(const oflow_image &img, void *dst, size_t elem, cudaStream_t s);
// Copies a dense device plane out to a caller buffer (host or device, pitch).
void unstage_plane(const float *src, int w, int h, float *dst, int pitch, int loc,
                   cudaStream_t s);
size_t dtype_size(int dtype);
void check_image(const oflow_image *img, const char *name);

}  // namespace oflow
