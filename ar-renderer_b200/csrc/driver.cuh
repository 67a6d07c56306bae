// Shared parts of the path tracer's two drivers (render.cu: one scene per call; batch.cu: many
// scenes in one graph launch): the per-device wavefront state, its buffers, and the kernels both
// drivers launch besides those of wavefront.cuh.
#pragma once

#include <algorithm>
#include <memory>

#include "guide_host.h"
#include "wavefront.cuh"

namespace prb {

// Guide inputs for every path filed as guided (kClassGuided): shading point, shading normal and
// outgoing direction (the same quantities the shading kernel records for training), FP16 rows in
// the order of that class's queue.
// kBatch: every path reads its own render's scene (and scene bounds).
template <bool kBatch = false>
__global__ void __launch_bounds__(256) k_guide_features(DevScene s0, const DevScene *scenes, Paths P,
                                                        const int *counters, const int *classQ, int classCap,
                                                        __half *feat, int bands) {
    const int n = counters[kCntClass0 + kClassGuided];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int j = classQ[size_t(kClassGuided) * classCap + i];
        const DevScene &s = SceneOf<kBatch>::get(s0, scenes, kBatch ? path_render(P.meta[j].w) : 0);
        const float *bmin = s.root.box, *bmax = s.root.box + 3;
        float4 o4 = P.o[j], d4 = P.d[j], hit = P.hit[j];
        V3 o = mk(o4.x, o4.y, o4.z), d = mk(d4.x, d4.y, d4.z);
        const prgpu::Primitive &pr = s.prims[__float_as_int(hit.w)];
        Surf sf = shade_point(s, pr, hit.x, hit.y, hit.z, o, d);
        float xn[3] = {(sf.p.x - bmin[0]) / fmaxf(bmax[0] - bmin[0], 1e-20f),
                       (sf.p.y - bmin[1]) / fmaxf(bmax[1] - bmin[1], 1e-20f),
                       (sf.p.z - bmin[2]) / fmaxf(bmax[2] - bmin[2], 1e-20f)};
        float f[kGuideIn];
#pragma unroll
        for (int k = 0; k < kGuideIn; ++k) f[k] = 0.f;
        guide_features_n(xn, sf.ns, -d, f, bands);
        guide_store_features(feat + size_t(i) * kGuideIn, f);
    }
}

// Order in which the collection visits a chunk's paths: warp-sized groups of consecutive paths,
// taken round-robin from kCollectSlices equal slices of the chunk (a transposition, so every path
// is visited once; t runs over [0, collect_span(total)) and j >= total is skipped). Paths are
// ordered sample-major, pixel-minor, and only the first `cap` samples are kept: visited in path
// order, those would all come from the first pixels of the image (its top rows on a large film).
constexpr int kCollectSlices = 1024;
__host__ __device__ __forceinline__ int collect_span(int total) {
    const int groups = (total + 31) >> 5;
    return ((groups + kCollectSlices - 1) / kCollectSlices) * kCollectSlices * 32;
}
__device__ __forceinline__ int collect_path(int t, int total) {
    const int groups = (total + 31) >> 5;
    const int per = (groups + kCollectSlices - 1) / kCollectSlices;
    const int g = t >> 5;
    return (((g % kCollectSlices) * per + g / kCollectSlices) << 5) | (t & 31);
}

// After a chunk's film: every complete training record of the chunk's paths becomes a sample
// (weight = (final mean radiance - snapshot) / mean throughput before the vertex), up to cap;
// every record is cleared for the next chunk.
__device__ __forceinline__ void guide_collect_path(const Paths &P, float4 *rec, int j, GuideTrainRec *out, int *count,
                                                   int cap) {
    const float4 L = P.L[j];
    const float Lavg = 0.25f * (L.x + L.y + L.z + L.w);
    for (int v = 0; v < kGuideVertices; ++v) {
        float4 *r = rec + 4 * (size_t(j) * kGuideVertices + v);
        float4 r3 = r[3];
        if (__float_as_int(r3.w) == 0) break;
        if (__float_as_int(r3.w) == 2) {
            float4 r0 = r[0], r1 = r[1], r2 = r[2];
            float w = r0.w > 0.f ? (Lavg - r2.w) / r0.w : 0.f;
            if (w > 0.f && isfinite(w)) {
                int k = atomicAdd(count, 1);
                if (k < cap) out[k] = GuideTrainRec{{r0.x, r0.y, r0.z}, {r1.x, r1.y, r1.z}, {r2.x, r2.y, r2.z},
                                                     {r3.x, r3.y, r3.z}, r1.w, w};
            }
        }
        r[3] = make_float4(0.f, 0.f, 0.f, __int_as_float(0));
    }
}

constexpr int kGuideBatch = 1 << 16;    // training samples per online step
constexpr int kGuideRecords = 1 << 18;  // samples kept per chunk: up to 4 steps

constexpr int kBouncesPerPoll = 4;  // bounces enqueued between two host reads of the queue length

struct RenderState {
    SceneCache scene;
    DevBuf pathBuf, shadowBuf, queues, classQueues, counters, stats, film;
    DevBuf guideFeat, guideOut, guideRec, guideTrain;  // guided form (allocated on first use)
    DevBuf sceneTable;  // the render's DevScene in device memory, for the shading kernels
    DevBuf tap;         // measurement tap (allocated on first use)
    int guideCap = 0;
    int capacity = 0;
    Paths P{};
    Shadows S{};
    int *hostActive = nullptr;          // pinned: the active-queue length, polled between bounce blocks
    cudaEvent_t ev[4 * kBouncesPerPoll + 2] = {};
    bool events = false;
    int residentExtend[2] = {0, 0}, residentShadow[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

// The guided form's per-path buffers for the state's capacity: FP16 features and FP32 network
// outputs per diffuse-queue entry, the training records per path (zeroed), and the samples of a
// chunk followed by their count.
void ensure_guide_buffers(RenderState &rs, cudaStream_t st);
GuideTrainRec *guide_train_recs(RenderState &rs);
int *guide_train_count(RenderState &rs);
// Path state, shadow queue, ray queues, class queues and counters for `cap` paths in flight.
void ensure_capacity(RenderState &rs, int cap);
// Blocks of 256 for `work` items, at most perSm per SM.
int grid_for(const DeviceState &ds, int64_t work, int perSm = 8);
// The per-device state of the single-render driver.
RenderState &render_state(int device);

template <typename K> int resident_blocks_of(K kernel) {
    int n = 0;
    PRB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, 256, 0));
    return std::max(1, n);
}

} // namespace prb
