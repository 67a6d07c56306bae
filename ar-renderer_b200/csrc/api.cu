// Module-level entry points: version queries, device listing, launch accounting and the
// per-device state behind every other entry point. Layout checks pin the v4 structs to the byte
// offsets of src/gpu/gpu_api.h so that a reference host can pass its own structs unchanged.

#include <cstring>
#include <cstddef>
#include <memory>
#include <vector>

#include "device.cuh"
#include "../../include/prgpu_api.h"
#include "guide.cuh"

namespace prb {

std::mutex gApiMutex;
std::atomic<uint64_t> gLaunchCount{0};

namespace {
std::vector<std::unique_ptr<DeviceState>> gStates;
int gDeviceCount = -1;
} // namespace

DeviceState &device_state(int deviceIndex) {
    if (gDeviceCount < 0) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess) {
            cudaGetLastError();
            n = 0;
        }
        gDeviceCount = n;
        gStates.resize(size_t(n));
    }
    if (deviceIndex < 0 || deviceIndex >= gDeviceCount) throw CudaError{"no such GPU device"};
    PRB_CUDA(cudaSetDevice(deviceIndex));
    auto &st = gStates[size_t(deviceIndex)];
    if (!st) {
        auto s = std::make_unique<DeviceState>();
        s->device = deviceIndex;
        PRB_CUDA(cudaGetDeviceProperties(&s->prop, deviceIndex));
        PRB_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        PRB_CUDA(cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking));
        st = std::move(s);
    }
    return *st;
}

} // namespace prb

// Byte layout of the v4 interface (x86-64 / aarch64 LP64), as compiled from src/gpu/gpu_api.h.
static_assert(sizeof(prgpu::Float3) == 12);
static_assert(sizeof(prgpu::Spectrum) == 380);
static_assert(sizeof(prgpu::BVHNode) == 32 && offsetof(prgpu::BVHNode, offset) == 24 &&
              offsetof(prgpu::BVHNode, nPrims) == 28 && offsetof(prgpu::BVHNode, axis) == 30);
static_assert(sizeof(prgpu::Primitive) == 128 && offsetof(prgpu::Primitive, p0) == 24 &&
              offsetof(prgpu::Primitive, n0) == 60 && offsetof(prgpu::Primitive, u0) == 96 &&
              offsetof(prgpu::Primitive, r) == 120);
static_assert(sizeof(prgpu::Material) == 88 && offsetof(prgpu::Material, coatEta) == 40 &&
              offsetof(prgpu::Material, sheenColor) == 72);
static_assert(sizeof(prgpu::Medium) == 16);
static_assert(sizeof(prgpu::Filter) == 276);
static_assert(sizeof(prgpu::Light) == 48 && offsetof(prgpu::Light, position) == 16 &&
              offsetof(prgpu::Light, pmf) == 40);
static_assert(sizeof(prgpu::Camera) == 80 && offsetof(prgpu::Camera, width) == 64);
static_assert(sizeof(prgpu::GridMediumDesc) == 160 && offsetof(prgpu::GridMediumDesc, density) == 104 &&
              offsetof(prgpu::GridMediumDesc, field) == 112);
static_assert(sizeof(prgpu::SceneExt) == 144 && offsetof(prgpu::SceneExt, rayTap) == 128 && offsetof(prgpu::SceneExt, gridMedia) == 40 &&
              offsetof(prgpu::SceneExt, sun) == 56 && offsetof(prgpu::SceneExt, deltaLights) == 72 &&
              offsetof(prgpu::SceneExt, rgbToSpectrum) == 104 && offsetof(prgpu::SceneExt, textureNodes) == 112);
static_assert(sizeof(prgpu::TextureNode) == 64);
static_assert(sizeof(prgpu::ImageTextureDesc) == 56 && sizeof(prgpu::MaterialTextures) == 72);
static_assert(sizeof(prgpu::DeltaLightDesc) == 104 && offsetof(prgpu::DeltaLightDesc, frame) == 48 &&
              offsetof(prgpu::DeltaLightDesc, profile) == 96);
static_assert(sizeof(prgpu::EnvMapDesc) == 32 && sizeof(prgpu::SunDesc) == 28);
static_assert(prgpu::kGuideParams == prb::kGuideParams);
static_assert(sizeof(prgpu::BatchItem) == 48 && offsetof(prgpu::BatchItem, outXYZ) == 40 &&
              sizeof(prgpu::BatchConfig) == 16 && sizeof(prgpu::BatchStats) == 72);
static_assert(sizeof(prgpu::RenderParams) == 24 && offsetof(prgpu::RenderParams, seed) == 8);
static_assert(sizeof(prgpu::DeviceInfo) == 304 && offsetof(prgpu::DeviceInfo, globalMemory) == 256);
static_assert(offsetof(prgpu::SceneDesc, nodes) == 8 && offsetof(prgpu::SceneDesc, cameraMedium) == 108 &&
              offsetof(prgpu::SceneDesc, camera) == 140 && offsetof(prgpu::SceneDesc, filter) == 220 &&
              offsetof(prgpu::SceneDesc, sheenAlbedo) == 496 && offsetof(prgpu::SceneDesc, cieYIntegral) == 512 &&
              sizeof(prgpu::SceneDesc) == 520);
static_assert(sizeof(prgpu::Ray) == 32);

using namespace prb;

PRGPU_API int prgpu_api_version() { return prgpu::kApiVersion; }

PRGPU_API int prgpu_ext_version() { return prgpu::kExtVersion; }

namespace prb {
std::vector<float> sheen_albedo_table();
}

PRGPU_API void prgpu_sheen_albedo_table(float *out) {
    if (!out) return;
    std::vector<float> t = prb::sheen_albedo_table();
    std::memcpy(out, t.data(), t.size() * sizeof(float));
}

PRGPU_API uint64_t prgpu_launch_count() { return gLaunchCount.load(); }

PRGPU_API int prgpu_list_devices(prgpu::DeviceInfo *out, int max) {
    std::lock_guard<std::mutex> lock(gApiMutex);
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int written = 0;
    for (int i = 0; i < n && written < max && out; ++i) {
        cudaDeviceProp p{};
        if (cudaGetDeviceProperties(&p, i) != cudaSuccess) continue;
        prgpu::DeviceInfo &d = out[written++];
        std::memset(&d, 0, sizeof(d));
        std::snprintf(d.name, sizeof(d.name), "%s", p.name);
        d.globalMemory = uint64_t(p.totalGlobalMem);
        d.computeUnits = p.multiProcessorCount;
        d.isGpu = 1;
        std::snprintf(d.backend, sizeof(d.backend), "cuda sm_%d%d", p.major, p.minor);
    }
    return written;
}
