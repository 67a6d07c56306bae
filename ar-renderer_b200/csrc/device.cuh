// Per-device runtime state shared by the entry points of libprender_gpu: device selection,
// streams, grow-only scratch buffers, error reporting and launch accounting. All entry points
// serialise on one mutex, as the reference module does (src/gpu/prender_gpu.cpp:1576, 1638).
#pragma once

#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace prb {

extern std::mutex gApiMutex;
extern std::atomic<uint64_t> gLaunchCount;

struct CudaError {
    std::string msg;
};

inline void check_cuda(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw CudaError{std::string(what) + ": " + cudaGetErrorString(e)};
}
#define PRB_CUDA(x) ::prb::check_cuda((x), #x)

inline void set_err(char *err, int len, const std::string &m) {
    if (err && len > 0) std::snprintf(err, size_t(len), "%s", m.c_str());
}

// Grow-only device buffer.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    void ensure(size_t n) {
        if (n <= bytes) return;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        PRB_CUDA(cudaMalloc(&ptr, n));
        bytes = n;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    template <typename T> T *as() const { return static_cast<T *>(ptr); }
};

struct DeviceState {
    int device = -1;
    cudaStream_t stream = nullptr;   // compute
    cudaStream_t copy = nullptr;     // host<->device copies overlapped with compute
    cudaDeviceProp prop{};
};

// Makes deviceIndex current and returns its state (created on first use); throws on failure.
DeviceState &device_state(int deviceIndex);

inline void count_launch(uint64_t n = 1) { gLaunchCount.fetch_add(n, std::memory_order_relaxed); }

} // namespace prb
