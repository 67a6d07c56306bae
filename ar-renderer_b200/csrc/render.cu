// Wavefront spectral volumetric path tracer: the drivers of the kernels in wavefront.cuh.
//   * prgpu_render / prgpu_render_ex: one scene per call, the host polling the active-queue length
//     once every few bounces;
//   * prgpu_render_batch: many scenes in one wavefront, run by one CUDA graph launch whose
//     device-side loop needs no host round trip, with settings from an autotuner.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>
#include <memory>

#include "guide_host.h"
#include "wavefront.cuh"
#include "aov.cuh"

namespace prb {
// ---------------------------------------------------------------------------------------------
// Driver

// Guide inputs for every path filed as diffuse: shading point, shading normal and outgoing
// direction (the same quantities the shading kernel records for training), FP16 rows in the
// order of the diffuse class queue.
__global__ void __launch_bounds__(256) k_guide_features(DevScene s, Paths P, const int *counters, const int *classQ,
                                                        int classCap, __half *feat) {
    const int n = counters[kCntClass0 + kClassDiffuse];
    const float *bmin = s.root.box, *bmax = s.root.box + 3;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int j = classQ[size_t(kClassDiffuse) * classCap + i];
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
        guide_features_n(xn, sf.ns, -d, f);
        __half2 *dst = reinterpret_cast<__half2 *>(feat + size_t(i) * kGuideIn);
#pragma unroll
        for (int k = 0; k < kGuideIn / 2; ++k) dst[k] = __floats2half2_rn(f[2 * k], f[2 * k + 1]);
    }
}

// After a chunk's film: every complete training record of the chunk's paths becomes a sample
// (weight = (final mean radiance - snapshot) / mean throughput before the vertex), up to cap;
// every record is cleared for the next chunk.
__global__ void __launch_bounds__(256) k_guide_collect(Paths P, float4 *rec, int total, GuideTrainRec *out,
                                                       int *count, int cap) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < total; j += gridDim.x * blockDim.x) {
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
}

// Measurement tap: the closest-hit rays of queued paths in slots [0, paths), then (before the
// shadow pass) the shadow rays, as 8-float records (origin, tMax, direction, 1) at bounce b.
__global__ void __launch_bounds__(256) k_tap_closest(Paths P, const int *counters, const int *queue, float4 *tap,
                                                     int paths, int bounce) {
    const int n = counters[kCntActive];
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int j = queue[q];
        if (j >= paths) continue;
        const float4 o = P.o[j], d = P.d[j];
        float4 *r = tap + 2 * (size_t(bounce) * paths + j);
        r[0] = make_float4(o.x, o.y, o.z, kInf);
        r[1] = make_float4(d.x, d.y, d.z, 1.f);
    }
}

__global__ void __launch_bounds__(256) k_tap_shadow(Shadows S, const int *counters, float4 *tap, int paths,
                                                    int bounces, int bounce) {
    const int n = counters[kCntShadow];
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const float4 o = S.o[q], d = S.d[q];
        const int j = __float_as_int(d.w);
        if (j < 0 || j >= paths) continue;
        float4 *r = tap + 2 * ((size_t(bounces) + bounce) * paths + j);
        r[0] = make_float4(o.x, o.y, o.z, 1.f - kShadowEps);
        r[1] = make_float4(d.x, d.y, d.z, 1.f);
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

std::unique_ptr<RenderState> gRender[64];

size_t carve(char *&p, size_t bytes) {
    size_t aligned = (bytes + 255) & ~size_t(255);
    p += aligned;
    return aligned;
}

void ensure_capacity(RenderState &rs, int cap) {
    if (rs.capacity >= cap) return;
    size_t perPath = 11 * sizeof(float4) + sizeof(ulonglong2) + sizeof(int4) + 256;
    rs.pathBuf.ensure(size_t(cap) * perPath + 16 * 256);
    char *base = rs.pathBuf.as<char>(), *p = base;
    auto take = [&](size_t bytes) {
        char *q = p;
        carve(p, bytes);
        return q;
    };
    rs.P.o = reinterpret_cast<float4 *>(take(cap * sizeof(float4)));
    rs.P.d = reinterpret_cast<float4 *>(take(cap * sizeof(float4)));
    rs.P.beta = reinterpret_cast<float4 *>(take(cap * sizeof(float4)));
    rs.P.rpath = reinterpret_cast<float4 *>(take(cap * sizeof(float4)));
    rs.P.L = reinterpret_cast<float4 *>(take(cap * sizeof(float4)));
    rs.P.Lhero = reinterpret_cast<float4 *>(take(cap * sizeof(float4)));
    rs.P.lam = reinterpret_cast<float4 *>(take(cap * sizeof(float4)));
    rs.P.lpdf = reinterpret_cast<float4 *>(take(cap * sizeof(float4)));
    rs.P.prevP = reinterpret_cast<float4 *>(take(cap * sizeof(float4)));
    rs.P.prevN = reinterpret_cast<float4 *>(take(cap * sizeof(float4)));
    rs.P.hit = reinterpret_cast<float4 *>(take(cap * sizeof(float4)));
    rs.P.rng = reinterpret_cast<ulonglong2 *>(take(cap * sizeof(ulonglong2)));
    rs.P.meta = reinterpret_cast<int4 *>(take(cap * sizeof(int4)));
    rs.shadowBuf.ensure(size_t(cap) * (3 * sizeof(float4) + sizeof(float)) + 8 * 256);
    p = rs.shadowBuf.as<char>();
    rs.S.o = reinterpret_cast<float4 *>(take(cap * sizeof(float4)));
    rs.S.d = reinterpret_cast<float4 *>(take(cap * sizeof(float4)));
    rs.S.c = reinterpret_cast<float4 *>(take(cap * sizeof(float4)));
    rs.S.w = reinterpret_cast<float *>(take(cap * sizeof(float)));
    rs.queues.ensure(size_t(2) * cap * sizeof(int));
    rs.classQueues.ensure(size_t(kClasses) * cap * sizeof(int));
    // The interface walk's queue reuses the class queues: they are dead between shading and the
    // next closest-hit pass, and a bounce queues at most one shadow entry per path.
    rs.S.walk = rs.classQueues.as<int>();
    rs.counters.ensure(kCntSlots * sizeof(int));
    rs.stats.ensure(kStatSlots * sizeof(unsigned long long));
    rs.capacity = cap;
}

int grid_for(const DeviceState &ds, int64_t work, int perSm = 8) {
    int64_t blocks = (work + 255) / 256;
    return int(std::max<int64_t>(1, std::min<int64_t>(blocks, int64_t(ds.prop.multiProcessorCount) * perSm)));
}

using ShadowAnyFn = void (*)(DevScene, const DevScene *, Paths, Shadows, int *);

// variant bit 0: spheres present, bit 1: media present, bit 2: medium interfaces present.
ShadowAnyFn shadow_any_kernel(int variant) {
    if (variant & 4) return (variant & 1) ? k_shadow_any<true, true, false, true> : k_shadow_any<false, true, false, true>;
    switch (variant & 3) {
    case 0: return k_shadow_any<false, false>;
    case 1: return k_shadow_any<true, false>;
    case 2: return k_shadow_any<false, true>;
    default: return k_shadow_any<true, true>;
    }
}

template <typename K> int resident_blocks_of(K kernel) {
    int n = 0;
    PRB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, 256, 0));
    return std::max(1, n);
}

// Renders params->spp samples of every pixel and adds them, in sample order, onto the device
// FP64 film rs.film (already initialised by the caller). Bounces are enqueued in blocks of
// kBouncesPerPoll with the queue advanced on the device; the host reads the queue length once
// per block to stop.
bool render_into_film(DeviceState &ds, RenderState &rs, const prgpu::RenderParams &rp, const prgpu::SceneExt *ext,
                      prgpu::RenderStats *stats, std::string *err) {
    cudaStream_t st = ds.stream;
    const DevScene &scene = rs.scene.ds;
    const int w = scene.cam.width, h = scene.cam.height;
    const int64_t npix = int64_t(w) * h;
    int pathTarget = (ext && ext->wavefrontPaths > 0) ? ext->wavefrontPaths : (1 << 21);
    pathTarget = std::max(pathTarget, 1024);
    int spp = rp.spp;
    if (spp <= 0) return true;
    int npixChunk = int(std::min<int64_t>(npix, pathTarget));
    int S = std::max(1, std::min(spp, pathTarget / npixChunk));
    ensure_capacity(rs, npixChunk * S);
    // The shading kernels read the scene from device memory, as the batched form does: their
    // out-of-line helpers then take it by pointer instead of copying the kernel parameter.
    rs.sceneTable.ensure(sizeof(DevScene));
    PRB_CUDA(cudaMemcpyAsync(rs.sceneTable.ptr, &scene, sizeof(DevScene), cudaMemcpyHostToDevice, st));
    if (!rs.events) {
        for (auto &e : rs.ev) PRB_CUDA(cudaEventCreate(&e));
        PRB_CUDA(cudaMallocHost(&rs.hostActive, sizeof(int)));
        rs.residentExtend[0] = resident_blocks_of(k_extend<false>);
        rs.residentExtend[1] = resident_blocks_of(k_extend<true>);
        for (int v = 0; v < 8; ++v) rs.residentShadow[v] = resident_blocks_of(shadow_any_kernel(v));
        rs.events = true;
    }
    int *cnt = rs.counters.as<int>();
    auto *dstats = rs.stats.as<unsigned long long>();
    int *qa = rs.queues.as<int>(), *qb = qa + rs.capacity;
    int *cq = rs.classQueues.as<int>();
    double traceMs = 0, shadeMs = 0, shadowMs = 0, filmMs = 0;
    uint64_t launches = 0;
    const int sph = rs.scene.hasSpheres ? 1 : 0;
    const int sms = ds.prop.multiProcessorCount;
    const int shadowVariant =
        sph | (scene.mediumCount + scene.gridCount > 0 ? 2 : 0) | (scene.hasInterfaces ? 6 : 0);
    const ShadowAnyFn shadowAny = shadow_any_kernel(shadowVariant);
    const int gExtend = sms * rs.residentExtend[sph], gShadow = sms * rs.residentShadow[shadowVariant];
    const int gShade = sms * 8;
    const bool timing = stats != nullptr;
    // Guided form: SceneExt::flags bit 0 samples diffuse vertices with the guide network, bit 1
    // trains it online (one Adam step per chunk on the chunk's recorded samples), bit 2 starts
    // from fresh weights.
    const int gflags = ext ? ext->flags : 0;
    const int guideMode = gflags & 3;
    GuideTrainRec *trainRecs = nullptr;
    int *trainCount = nullptr;
    GuideOpts gopts;
    if (guideMode) {
        guide_prepare(ds, ds.device, (gflags & 4) != 0, rp.seed);
        gopts = guide_options(ds.device);
        if (rs.guideCap < rs.capacity) {
            rs.guideFeat.ensure(size_t(rs.capacity) * kGuideIn * sizeof(__half));
            rs.guideOut.ensure(size_t(rs.capacity) * kGuideOut * sizeof(float));
            const size_t recBytes = size_t(rs.capacity) * kGuideVertices * 4 * sizeof(float4);
            rs.guideRec.ensure(recBytes);
            PRB_CUDA(cudaMemsetAsync(rs.guideRec.ptr, 0, recBytes, st));
            rs.guideTrain.ensure(size_t(kGuideRecords) * sizeof(GuideTrainRec) + 256);
            rs.guideCap = rs.capacity;
        }
        trainRecs = rs.guideTrain.as<GuideTrainRec>();
        trainCount = reinterpret_cast<int *>(rs.guideTrain.as<unsigned char>() + size_t(kGuideRecords) * sizeof(GuideTrainRec));
    }
    // Measurement tap of the first chunk's rays (SceneExt::rayTap).
    const int tapPaths = (ext && ext->rayTap) ? std::max(0, ext->rayTapPaths) : 0;
    const int tapBounces = tapPaths > 0 ? std::max(0, ext->rayTapBounces) : 0;
    const size_t tapBytes = size_t(2) * tapBounces * tapPaths * 8 * sizeof(float);
    if (tapBytes) {
        rs.tap.ensure(tapBytes);
        PRB_CUDA(cudaMemsetAsync(rs.tap.ptr, 0, tapBytes, st));
    }
    int bounceIndex = 0;
    PRB_CUDA(cudaMemsetAsync(cnt, 0, kCntSlots * sizeof(int), st));
    PRB_CUDA(cudaMemsetAsync(dstats, 0, kStatSlots * sizeof(unsigned long long), st));
    for (int64_t pix0 = 0; pix0 < npix; pix0 += npixChunk) {
        int np = int(std::min<int64_t>(npixChunk, npix - pix0));
        for (int s0 = 0; s0 < spp; s0 += S) {
            ChunkInfo ci;
            ci.pixBegin = int(pix0);
            ci.npix = np;
            ci.samples = std::min(S, spp - s0);
            ci.firstSample = rp.firstSample + s0;
            ci.seed = rp.seed;
            ci.maxDepth = rp.maxDepth;
            int total = np * ci.samples;
            k_raygen<<<grid_for(ds, total), 256, 0, st>>>(scene, rs.P, ci, cnt, qa);
            ++launches;
            int *qin = qa, *qout = qb;
            for (;;) {
                for (int b = 0; b < kBouncesPerPoll; ++b) {
                    const bool tapNow = tapBytes && pix0 == 0 && s0 == 0 && bounceIndex < tapBounces;
                    if (tapNow) {
                        k_tap_closest<<<gShade, 256, 0, st>>>(rs.P, cnt, qin, rs.tap.as<float4>(), tapPaths, bounceIndex);
                        ++launches;
                    }
                    if (timing) PRB_CUDA(cudaEventRecord(rs.ev[4 * b], st));
                    if (sph) k_extend<true><<<gExtend, 256, 0, st>>>(scene, nullptr, rs.P, cnt, qin);
                    else k_extend<false><<<gExtend, 256, 0, st>>>(scene, nullptr, rs.P, cnt, qin);
                    k_classify<false><<<gShade, 256, 0, st>>>(scene, nullptr, rs.P, cnt, qin, cq, rs.capacity);
                    if (guideMode & 1) {
                        k_guide_features<<<gShade, 256, 0, st>>>(scene, rs.P, cnt, cq, rs.capacity,
                                                                 rs.guideFeat.as<__half>());
                        guide_infer_rows(st, ds.device, rs.guideFeat.as<__half>(), cnt + kCntClass0 + kClassDiffuse,
                                         rs.capacity, rs.guideOut.as<float>());
                        launches += 1 + kGuideInferLaunches;
                    }
                    if (timing) PRB_CUDA(cudaEventRecord(rs.ev[4 * b + 1], st));
                    ShadeArgs sa{scene, rs.sceneTable.as<DevScene>(), rs.P, rs.S, cq, rs.capacity, qout, cnt,
                                 rp.maxDepth, 0, rs.guideOut.as<float>(), rs.guideRec.as<float4>(), guideMode, qin,
                                 gopts};
                    const bool dl = scene.deltaCount > 0 || scene.matTex != nullptr;
                    if (guideMode) {
                        if (dl) k_shade<false, true, false, true><<<gShade, 256, 0, st>>>(sa);
                        else k_shade<false, true><<<gShade, 256, 0, st>>>(sa);
                    } else {
                        if (dl) k_shade<false, false, false, true><<<gShade, 256, 0, st>>>(sa);
                        else k_shade<false, false><<<gShade, 256, 0, st>>>(sa);
                    }
                    if (scene.hasFull) {
                        if (dl) k_shade<false, false, true, true><<<gShade, 256, 0, st>>>(sa);
                        else k_shade<false, false, true><<<gShade, 256, 0, st>>>(sa);
                        ++launches;
                    }
                    if (tapNow) {
                        k_tap_shadow<<<gShade, 256, 0, st>>>(rs.S, cnt, rs.tap.as<float4>(), tapPaths, tapBounces,
                                                             bounceIndex);
                        ++launches;
                    }
                    ++bounceIndex;
                    if (timing) PRB_CUDA(cudaEventRecord(rs.ev[4 * b + 2], st));
                    shadowAny<<<gShadow, 256, 0, st>>>(scene, nullptr, rs.P, rs.S, cnt);
                    if (scene.hasInterfaces) {
                        if (sph) k_shadow_walk<true><<<gShade, 256, 0, st>>>(scene, nullptr, rs.P, rs.S, cnt);
                        else k_shadow_walk<false><<<gShade, 256, 0, st>>>(scene, nullptr, rs.P, rs.S, cnt);
                        ++launches;
                    }
                    if (timing) PRB_CUDA(cudaEventRecord(rs.ev[4 * b + 3], st));
                    k_advance<<<1, 1, 0, st>>>(cnt, dstats);
                    launches += 5;
                    std::swap(qin, qout);
                }
                PRB_CUDA(cudaGetLastError());
                PRB_CUDA(cudaMemcpyAsync(rs.hostActive, cnt + kCntActive, sizeof(int), cudaMemcpyDeviceToHost, st));
                PRB_CUDA(cudaStreamSynchronize(st));
                if (timing) {
                    for (int b = 0; b < kBouncesPerPoll; ++b) {
                        float x = 0, y = 0, z = 0;
                        PRB_CUDA(cudaEventElapsedTime(&x, rs.ev[4 * b], rs.ev[4 * b + 1]));
                        PRB_CUDA(cudaEventElapsedTime(&y, rs.ev[4 * b + 1], rs.ev[4 * b + 2]));
                        PRB_CUDA(cudaEventElapsedTime(&z, rs.ev[4 * b + 2], rs.ev[4 * b + 3]));
                        traceMs += x;
                        shadeMs += y;
                        shadowMs += z;
                    }
                }
                if (*rs.hostActive == 0) break;
            }
            if (timing) PRB_CUDA(cudaEventRecord(rs.ev[4 * kBouncesPerPoll], st));
            k_film<<<grid_for(ds, np), 256, 0, st>>>(scene, rs.P, ci, rp.clampLuminance, rs.film.as<double>());
            ++launches;
            if (guideMode & 2) {
                PRB_CUDA(cudaMemsetAsync(trainCount, 0, sizeof(int), st));
                k_guide_collect<<<grid_for(ds, total), 256, 0, st>>>(rs.P, rs.guideRec.as<float4>(), total, trainRecs,
                                                                     trainCount, kGuideRecords);
                for (int pass = 0; pass < gopts.trainPasses; ++pass)
                    for (int k = 0; k < kGuideRecords / kGuideBatch; ++k)
                        guide_train_records(st, ds.device, trainRecs, trainCount, k * kGuideBatch, kGuideBatch, 0.f);
                launches += 1 + gopts.trainPasses * (kGuideRecords / kGuideBatch) * kGuideTrainLaunches;
            }
            if (timing) {
                PRB_CUDA(cudaEventRecord(rs.ev[4 * kBouncesPerPoll + 1], st));
                PRB_CUDA(cudaEventSynchronize(rs.ev[4 * kBouncesPerPoll + 1]));
                float f = 0;
                PRB_CUDA(cudaEventElapsedTime(&f, rs.ev[4 * kBouncesPerPoll], rs.ev[4 * kBouncesPerPoll + 1]));
                filmMs += f;
            }
        }
    }
    PRB_CUDA(cudaGetLastError());
    int status = 0;
    unsigned long long hs[kStatSlots] = {};
    PRB_CUDA(cudaMemcpyAsync(&status, cnt + kCntStatus, sizeof(int), cudaMemcpyDeviceToHost, st));
    PRB_CUDA(cudaMemcpyAsync(hs, dstats, sizeof(hs), cudaMemcpyDeviceToHost, st));
    if (tapBytes) PRB_CUDA(cudaMemcpyAsync(ext->rayTap, rs.tap.ptr, tapBytes, cudaMemcpyDeviceToHost, st));
    PRB_CUDA(cudaStreamSynchronize(st));
    count_launch(launches);
    if (stats) {
        stats->pathSamples += uint64_t(npix) * uint64_t(spp);
        stats->closestRays += hs[kStatClosest];
        stats->shadowRays += hs[kStatShadow];
        stats->bounces += hs[kStatBounces];
        stats->kernelLaunches += launches;
        stats->traceMs += traceMs;
        stats->shadeMs += shadeMs;
        stats->shadowMs += shadowMs;
        stats->filmMs += filmMs;
    }
    if (status & kStatusStack) {
        *err = "BVH deeper than the traversal stack (64 entries)";
        return false;
    }
    if (guideMode && guide_failed(ds, ds.device)) {
        *err = "guide kernel timed out waiting for the tensor cores";
        return false;
    }
    // kStatusGuard: the 8,192-step guard of the reference ended some paths; not an error there either.
    return true;
}

RenderState &render_state(int device) {
    auto &p = gRender[device];
    if (!p) p = std::make_unique<RenderState>();
    return *p;
}

int render_common(int deviceIndex, const prgpu::SceneDesc *sd, const prgpu::SceneExt *ext,
                  const prgpu::RenderParams *params, float *outF, double *outD, prgpu::RenderStats *stats, char *err,
                  int errLen) {
    std::lock_guard<std::mutex> lock(gApiMutex);
    try {
        if (!sd || sd->apiVersion != prgpu::kApiVersion) {
            set_err(err, errLen, "API version mismatch");
            return 1;
        }
        if (!params || params->spp < 0) {
            set_err(err, errLen, "bad render parameters");
            return 1;
        }
        if (ext && ext->structSize != sizeof(prgpu::SceneExt)) {
            set_err(err, errLen, "SceneExt size mismatch");
            return 1;
        }
        if (deviceIndex < 0 || deviceIndex >= 64) {
            set_err(err, errLen, "no such GPU device");
            return 1;
        }
        DeviceState &ds = device_state(deviceIndex);
        RenderState &rs = render_state(deviceIndex);
        std::string e;
        if (!upload_scene(ds, sd, ext, rs.scene, &e)) {
            set_err(err, errLen, e);
            return 1;
        }
        const size_t n = size_t(sd->camera.width) * size_t(sd->camera.height) * 3;
        rs.film.ensure(n * sizeof(double));
        cudaEvent_t t0, t1;
        PRB_CUDA(cudaEventCreate(&t0));
        PRB_CUDA(cudaEventCreate(&t1));
        if (outD)
            PRB_CUDA(cudaMemcpyAsync(rs.film.ptr, outD, n * sizeof(double), cudaMemcpyHostToDevice, ds.stream));
        else
            PRB_CUDA(cudaMemsetAsync(rs.film.ptr, 0, n * sizeof(double), ds.stream));
        PRB_CUDA(cudaEventRecord(t0, ds.stream));
        if (stats) *stats = prgpu::RenderStats{};
        if (!render_into_film(ds, rs, *params, ext, stats, &e)) {
            set_err(err, errLen, e);
            return 1;
        }
        PRB_CUDA(cudaEventRecord(t1, ds.stream));
        if (outD) {
            PRB_CUDA(cudaMemcpyAsync(outD, rs.film.ptr, n * sizeof(double), cudaMemcpyDeviceToHost, ds.stream));
            PRB_CUDA(cudaStreamSynchronize(ds.stream));
        } else {
            std::vector<double> host(n);
            PRB_CUDA(cudaMemcpyAsync(host.data(), rs.film.ptr, n * sizeof(double), cudaMemcpyDeviceToHost, ds.stream));
            PRB_CUDA(cudaStreamSynchronize(ds.stream));
            for (size_t i = 0; i < n; ++i) outF[i] += float(host[i]);
        }
        if (stats) {
            float ms = 0;
            PRB_CUDA(cudaEventElapsedTime(&ms, t0, t1));
            stats->deviceMs = ms;
        }
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        return 0;
    } catch (const CudaError &ex) {
        set_err(err, errLen, ex.msg);
        return 1;
    } catch (const std::exception &ex) {
        set_err(err, errLen, ex.what());
        return 1;
    }
}

// ---------------------------------------------------------------------------------------------
// Batched renders (prgpu_render_batch): many scenes in one wavefront, one graph launch
//
// The host cuts every render into chunks (a pixel range x a sample range) and packs them into
// waves of at most half the path slots, at most one chunk per render per wave, so that one film
// kernel per wave can add each chunk's samples in sample order with no two chunks touching the same
// pixel. The device runs the waves from a conditional while node, two waves in flight: wave w
// lives in slot half w % 2, and as soon as a half is free the next wave is raygenned into it and
// joins the shared queues while the other wave's longest paths finish. Each iteration raygens (if
// a wave was started), advances every live path two bounces, films the oldest wave once its half
// has no live path left, and sets the loop condition. Waves are filmed strictly in order.

struct BatchChunk {
    int render, pixBegin, npix, samples;
    int firstSample, pathBase, pixBase, pad;
    uint64_t seed;
};
struct BatchWave {
    int firstChunk, nChunks, totalPaths, totalPix;
};
struct BatchCtl {
    int nWaves, nextWave, filmWave, iter, maxIter, status;
    int halfWave[2];      // wave occupying each slot half (-1: free)
    int rgHalf, rgWave;   // wave to raygen at the start of the next iteration (rgHalf -1: none)
    int halfSlots, pad;
};

constexpr int kMaxBatch = 256;  // render index in 8 bits of meta.w

// Largest chunk index i in [lo, lo + n) whose base (path or pixel prefix) is <= key.
__device__ __forceinline__ int find_chunk(const BatchChunk *c, int lo, int n, int key, bool byPixel) {
    int a = lo, b = lo + n - 1;
    while (a < b) {
        int m = (a + b + 1) >> 1;
        int v = byPixel ? c[m].pixBase : c[m].pathBase;
        if (v <= key) a = m;
        else b = m - 1;
    }
    return a;
}

__global__ void __launch_bounds__(256) k_batch_raygen(const DevScene *scenes, Paths P, const BatchCtl *ctl,
                                                      const BatchWave *waves, const BatchChunk *chunks, int *counters,
                                                      int *queue) {
    const int half = ctl->rgHalf;
    if (half < 0) return;
    const BatchWave w = waves[ctl->rgWave];
    const int base = half * ctl->halfSlots;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < w.totalPaths; j += gridDim.x * blockDim.x) {
        const BatchChunk &c = chunks[find_chunk(chunks, w.firstChunk, w.nChunks, j, false)];
        int local = j - c.pathBase, sIdx = local / c.npix, pl = local - sIdx * c.npix;
        raygen_path(scenes[c.render], P, base + j, c.pixBegin + pl, uint64_t(c.firstSample) + uint64_t(sIdx), c.seed,
                    c.render, counters, queue);
    }
}

// The slot half holding the oldest unfilmed wave if none of its paths is left, else -1. The film
// kernel and the loop control evaluate it on the same state.
__device__ __forceinline__ int half_to_film(const BatchCtl &c, const int *counters) {
    for (int h = 0; h < 2; ++h)
        if (c.halfWave[h] == c.filmWave && c.filmWave < c.nWaves && counters[kCntLive0 + h] == 0) return h;
    return -1;
}

__global__ void __launch_bounds__(256) k_batch_film(const DevScene *scenes, Paths P, const BatchCtl *ctl,
                                                    const BatchWave *waves, const BatchChunk *chunks,
                                                    const int *counters) {
    const BatchCtl c = *ctl;
    const int h = half_to_film(c, counters);
    if (h < 0) return;
    const BatchWave w = waves[c.filmWave];
    const int base = h * c.halfSlots;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < w.totalPix; t += gridDim.x * blockDim.x) {
        const BatchChunk &ch = chunks[find_chunk(chunks, w.firstChunk, w.nChunks, t, true)];
        const DevScene &s = scenes[ch.render];
        int pl = t - ch.pixBase;
        film_pixel(s, P, base + ch.pathBase, ch.npix, pl, ch.samples, s.clampY, s.film + 3 * size_t(ch.pixBegin + pl));
    }
}

// Loop control (one thread): retire the filmed wave, start the next wave in a free half, stop once
// the last wave is filmed -- or at the iteration bound (every path ends within 8,192 iterations of
// the shading guard, so the bound is only reached by a fault in this bookkeeping; status bit 0).
__global__ void k_batch_ctl(BatchCtl *ctl, const int *counters, cudaGraphConditionalHandle loop, int inGraph) {
    BatchCtl c = *ctl;
    ++c.iter;
    c.rgHalf = -1;
    const int h = half_to_film(c, counters);
    if (h >= 0) {
        c.halfWave[h] = -1;
        ++c.filmWave;
    }
    if (c.nextWave < c.nWaves) {
        int freeHalf = c.halfWave[0] < 0 ? 0 : (c.halfWave[1] < 0 ? 1 : -1);
        if (freeHalf >= 0) {
            c.halfWave[freeHalf] = c.nextWave;
            c.rgHalf = freeHalf;
            c.rgWave = c.nextWave;
            ++c.nextWave;
        }
    }
    unsigned more = c.filmWave < c.nWaves ? 1u : 0u;
    if (more && c.iter >= c.maxIter) {
        c.status |= 1;
        more = 0u;
    }
    *ctl = c;
    if (inGraph) cudaGraphSetConditional(loop, more);
}

__global__ void k_batch_init(BatchCtl *ctl, int nWaves, int maxIter, int halfSlots, int *counters,
                             unsigned long long *stats) {
    int i = threadIdx.x;
    if (i == 0) {
        BatchCtl c{};
        c.nWaves = nWaves;
        c.nextWave = 1;
        c.filmWave = 0;
        c.maxIter = maxIter;
        c.halfWave[0] = 0;
        c.halfWave[1] = -1;
        c.rgHalf = 0;
        c.rgWave = 0;
        c.halfSlots = halfSlots;
        *ctl = c;
    }
    if (i < kCntSlots) counters[i] = 0;
    if (i < kStatSlots) stats[i] = 0ull;
}

struct BatchGraphKey {
    int capacity = 0, shadeBlock = 0, variant = -1;
    const void *ptrs[7] = {};
    bool operator==(const BatchGraphKey &o) const {
        if (capacity != o.capacity || shadeBlock != o.shadeBlock || variant != o.variant) return false;
        for (int i = 0; i < 7; ++i)
            if (ptrs[i] != o.ptrs[i]) return false;
        return true;
    }
};

struct BatchState {
    std::vector<std::unique_ptr<SceneCache>> caches;
    RenderState paths;                  // path / shadow state, queues and counters (its scene unused)
    DevBuf scenes, chunks, waves, ctl, films;
    cudaGraphExec_t exec = nullptr;
    BatchGraphKey key;
    int64_t launchesPerIteration = 0;
    std::map<uint64_t, std::pair<int, int>> tuned;  // batch shape -> (wavefrontPaths, shadeBlock)
    cudaEvent_t ev[2] = {};
};

std::unique_ptr<BatchState> gBatch[64];

BatchState &batch_state(int device) {
    auto &p = gBatch[device];
    if (!p) {
        p = std::make_unique<BatchState>();
        PRB_CUDA(cudaEventCreate(&p->ev[0]));
        PRB_CUDA(cudaEventCreate(&p->ev[1]));
    }
    return *p;
}

// Packs the renders into waves (see the section comment), render-major: a wave takes the renders
// in index order, each as much as the remaining budget allows, so a wave touches few scenes and
// their BVHs stay in L2. Chunks of one render follow its sample order: whole frames of S samples
// while a frame fits the budget, else pixel ranges of one sample.
void schedule_waves(const std::vector<int64_t> &npix, const std::vector<int> &spp, int capacity,
                    const std::vector<prgpu::RenderParams> &rp, std::vector<BatchChunk> *chunks,
                    std::vector<BatchWave> *waves) {
    const int n = int(npix.size());
    std::vector<int64_t> nextPix(static_cast<size_t>(n), 0);
    std::vector<int> nextSample(static_cast<size_t>(n), 0);
    auto remaining = [&](int r) {
        return (int64_t(spp[size_t(r)]) - nextSample[size_t(r)]) * npix[size_t(r)] - nextPix[size_t(r)];
    };
    int first = 0;
    for (;;) {
        while (first < n && remaining(first) <= 0) ++first;
        if (first >= n) break;
        BatchWave w{int(chunks->size()), 0, 0, 0};
        int64_t budget = capacity;
        for (int r = first; r < n && budget > 0; ++r) {
            if (remaining(r) <= 0) continue;
            BatchChunk c{};
            c.render = r;
            c.seed = rp[size_t(r)].seed;
            const int64_t np = npix[size_t(r)];
            int64_t &pix = nextPix[size_t(r)];
            int &smp = nextSample[size_t(r)];
            if (pix == 0 && np <= budget) {
                int64_t S = std::min<int64_t>(spp[size_t(r)] - smp, budget / np);
                c.pixBegin = 0;
                c.npix = int(np);
                c.samples = int(S);
                c.firstSample = rp[size_t(r)].firstSample + smp;
                smp += int(S);
            } else {
                int64_t take = std::min<int64_t>(budget, np - pix);
                c.pixBegin = int(pix);
                c.npix = int(take);
                c.samples = 1;
                c.firstSample = rp[size_t(r)].firstSample + smp;
                pix += take;
                if (pix == np) {
                    pix = 0;
                    ++smp;
                }
            }
            c.pathBase = w.totalPaths;
            c.pixBase = w.totalPix;
            w.totalPaths += c.npix * c.samples;
            w.totalPix += c.npix;
            budget -= int64_t(c.npix) * c.samples;
            chunks->push_back(c);
            ++w.nChunks;
        }
        waves->push_back(w);
    }
}

uint64_t batch_shape_key(int device, int count, const prgpu::BatchItem *items) {
    uint64_t h = 1469598103934665603ull ^ uint64_t(device);
    auto mix = [&](uint64_t v) { h = (h ^ v) * 1099511628211ull; };
    mix(uint64_t(count));
    for (int i = 0; i < count; ++i) {
        const prgpu::SceneDesc *sd = items[i].scene;
        mix(uint64_t(sd->camera.width) << 32 | uint32_t(sd->camera.height));
        mix(uint64_t(items[i].params.spp) << 32 | uint32_t(items[i].params.maxDepth));
        mix(uint64_t(sd->primCount) << 32 | uint32_t(sd->mediumCount + (items[i].ext ? items[i].ext->gridMediumCount : 0)));
    }
    return h;
}

// Kernel launch shape of the loop body for one batch configuration.
struct BatchLaunch {
    void (*extend)(DevScene, const DevScene *, Paths, int *, const int *);
    void (*shadowAny)(DevScene, const DevScene *, Paths, Shadows, int *);
    void (*shadowWalk)(DevScene, const DevScene *, Paths, Shadows, int *);
    void (*shade)(ShadeArgs);
    void (*shadeFull)(ShadeArgs);
    bool walls, full;
    int gExtend, gShadow, gShade, gWide, shadeBlock, capacity;
};

BatchLaunch batch_launch(const DeviceState &ds, const BatchGraphKey &key) {
    const bool sph = key.variant & 1, media = key.variant & 2;
    BatchLaunch L{};
    L.walls = key.variant & 4;
    L.full = key.variant & 8;
    const bool dl = key.variant & 16;
    L.shade = dl ? k_shade<true, false, false, true> : k_shade<true>;
    L.shadeFull = dl ? k_shade<true, false, true, true> : k_shade<true, false, true>;
    L.extend = sph ? k_extend<true, true> : k_extend<false, true>;
    L.shadowAny = L.walls ? (sph ? k_shadow_any<true, true, true, true> : k_shadow_any<false, true, true, true>)
                  : sph   ? (media ? k_shadow_any<true, true, true> : k_shadow_any<true, false, true>)
                          : (media ? k_shadow_any<false, true, true> : k_shadow_any<false, false, true>);
    L.shadowWalk = sph ? k_shadow_walk<true, true> : k_shadow_walk<false, true>;
    const int sms = ds.prop.multiProcessorCount;
    L.gExtend = sms * resident_blocks_of(L.extend);
    L.gShadow = sms * resident_blocks_of(L.shadowAny);
    int perSm = 0;
    PRB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, L.shade, key.shadeBlock, 0));
    L.gShade = sms * std::max(1, perSm);
    L.gWide = sms * 8;
    L.shadeBlock = key.shadeBlock;
    L.capacity = key.capacity;
    return L;
}

// Enqueues one iteration of the batch loop on st (captured into the graph, or launched directly
// in the host-driven mode); returns the number of kernels.
int enqueue_batch_iteration(cudaStream_t st, BatchState &bs, const BatchLaunch &L, cudaGraphConditionalHandle loop,
                            bool inGraph) {
    RenderState &rs = bs.paths;
    const DevScene *scenes = bs.scenes.as<DevScene>();
    auto *ctl = bs.ctl.as<BatchCtl>();
    const auto *waves = bs.waves.as<BatchWave>();
    const auto *chunks = bs.chunks.as<BatchChunk>();
    int *cnt = rs.counters.as<int>();
    auto *dstats = rs.stats.as<unsigned long long>();
    int *qa = rs.queues.as<int>(), *qb = qa + L.capacity;
    int *cq = rs.classQueues.as<int>();
    DevScene none{};
    int launches = 0;
    k_batch_raygen<<<L.gWide, 256, 0, st>>>(scenes, rs.P, ctl, waves, chunks, cnt, qa);
    ++launches;
    int *qin = qa, *qout = qb;
    for (int b = 0; b < 2; ++b) {
        L.extend<<<L.gExtend, 256, 0, st>>>(none, scenes, rs.P, cnt, qin);
        k_classify<true><<<L.gWide, 256, 0, st>>>(none, scenes, rs.P, cnt, qin, cq, rs.capacity);
        ShadeArgs sa{none, scenes, rs.P, rs.S, cq, rs.capacity, qout, cnt, 0, L.capacity / 2, nullptr, nullptr, 0, qin};
        L.shade<<<L.gShade, L.shadeBlock, 0, st>>>(sa);
        if (L.full) {
            L.shadeFull<<<L.gShade, L.shadeBlock, 0, st>>>(sa);
            ++launches;
        }
        L.shadowAny<<<L.gShadow, 256, 0, st>>>(none, scenes, rs.P, rs.S, cnt);
        if (L.walls) {
            L.shadowWalk<<<L.gWide, 256, 0, st>>>(none, scenes, rs.P, rs.S, cnt);
            ++launches;
        }
        k_advance<<<1, 1, 0, st>>>(cnt, dstats);
        launches += 5;
        std::swap(qin, qout);
    }
    k_batch_film<<<L.gWide, 256, 0, st>>>(scenes, rs.P, ctl, waves, chunks, cnt);
    k_batch_ctl<<<1, 1, 0, st>>>(ctl, cnt, loop, inGraph ? 1 : 0);
    return launches + 2;
}

// Captures the loop body into the while node's body graph and instantiates the graph.
void build_batch_graph(DeviceState &ds, BatchState &bs, const BatchGraphKey &key) {
    if (bs.exec) {
        cudaGraphExecDestroy(bs.exec);
        bs.exec = nullptr;
    }
    const BatchLaunch L = batch_launch(ds, key);
    cudaStream_t st = ds.stream;
    cudaGraph_t g = nullptr;
    PRB_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle loop;
    PRB_CUDA(cudaGraphConditionalHandleCreate(&loop, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = loop;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    PRB_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    PRB_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    int launches = enqueue_batch_iteration(st, bs, L, loop, true);
    cudaGraph_t captured = nullptr;
    cudaError_t ce = cudaStreamEndCapture(st, &captured);
    if (ce != cudaSuccess) {
        cudaGraphDestroy(g);
        check_cuda(ce, "cudaStreamEndCapture");
    }
    cudaError_t ie = cudaGraphInstantiate(&bs.exec, g, 0);
    cudaGraphDestroy(g);
    check_cuda(ie, "cudaGraphInstantiate");
    bs.key = key;
    bs.launchesPerIteration = launches;
}

// One batch render with the given settings. trial: films start at zero on the device and are
// not copied back (autotuning). Returns false with a message on invalid input.
bool run_batch(DeviceState &ds, BatchState &bs, int count, const prgpu::BatchItem *items, int capacity, int shadeBlock,
               bool hostLoop, bool trial, int sppDivisor, prgpu::BatchStats *stats, std::string *err) {
    auto tHost0 = std::chrono::steady_clock::now();
    cudaStream_t st = ds.stream;
    if (int(bs.caches.size()) < count) bs.caches.resize(size_t(count));
    std::vector<int64_t> npix(static_cast<size_t>(count));
    std::vector<int> spp(static_cast<size_t>(count));
    std::vector<prgpu::RenderParams> rp(static_cast<size_t>(count));
    std::vector<size_t> filmOff(static_cast<size_t>(count));
    size_t filmTotal = 0;
    int sph = 0;
    bool media = false, walls = false, full = false, deltas = false;
    for (int i = 0; i < count; ++i) {
        if (!bs.caches[size_t(i)]) bs.caches[size_t(i)] = std::make_unique<SceneCache>();
        std::string e;
        if (!upload_scene(ds, items[i].scene, items[i].ext, *bs.caches[size_t(i)], &e)) {
            *err = "batch item " + std::to_string(i) + ": " + e;
            return false;
        }
        const DevScene &d = bs.caches[size_t(i)]->ds;
        npix[size_t(i)] = int64_t(d.cam.width) * d.cam.height;
        rp[size_t(i)] = items[i].params;
        spp[size_t(i)] = sppDivisor > 1 ? std::max(1, items[i].params.spp / sppDivisor) : items[i].params.spp;
        if (items[i].params.spp == 0) spp[size_t(i)] = 0;
        filmOff[size_t(i)] = filmTotal;
        filmTotal += size_t(npix[size_t(i)]) * 3;
        if (bs.caches[size_t(i)]->hasSpheres) sph = 1;
        if (d.mediumCount + d.gridCount > 0) media = true;
        if (d.hasInterfaces) walls = true;
        if (d.hasFull) full = true;
        if (d.deltaCount > 0 || d.matTex != nullptr) deltas = true;
    }
    std::vector<BatchChunk> chunks;
    std::vector<BatchWave> waves;
    schedule_waves(npix, spp, capacity / 2, rp, &chunks, &waves);
    ensure_capacity(bs.paths, capacity);
    bs.films.ensure(std::max<size_t>(1, filmTotal) * sizeof(double));
    bs.scenes.ensure(size_t(count) * sizeof(DevScene));
    bs.chunks.ensure(std::max<size_t>(1, chunks.size()) * sizeof(BatchChunk));
    bs.waves.ensure(std::max<size_t>(1, waves.size()) * sizeof(BatchWave));
    bs.ctl.ensure(sizeof(BatchCtl));
    double *films = bs.films.as<double>();
    std::vector<DevScene> table(static_cast<size_t>(count));
    for (int i = 0; i < count; ++i) {
        DevScene d = bs.caches[size_t(i)]->ds;
        d.maxDepth = items[i].params.maxDepth;
        d.clampY = items[i].params.clampLuminance;
        d.film = films + filmOff[size_t(i)];
        table[size_t(i)] = d;
        size_t bytes = size_t(npix[size_t(i)]) * 3 * sizeof(double);
        if (trial) PRB_CUDA(cudaMemsetAsync(d.film, 0, bytes, st));
        else PRB_CUDA(cudaMemcpyAsync(d.film, items[i].outXYZ, bytes, cudaMemcpyHostToDevice, st));
    }
    PRB_CUDA(cudaMemcpyAsync(bs.scenes.ptr, table.data(), table.size() * sizeof(DevScene), cudaMemcpyHostToDevice, st));
    if (!chunks.empty())
        PRB_CUDA(cudaMemcpyAsync(bs.chunks.ptr, chunks.data(), chunks.size() * sizeof(BatchChunk),
                                 cudaMemcpyHostToDevice, st));
    if (!waves.empty())
        PRB_CUDA(cudaMemcpyAsync(bs.waves.ptr, waves.data(), waves.size() * sizeof(BatchWave), cudaMemcpyHostToDevice,
                                 st));
    BatchGraphKey key;
    key.capacity = capacity;
    key.shadeBlock = shadeBlock;
    key.variant = sph | (media ? 2 : 0) | (walls ? 4 : 0) | (full ? 8 : 0) | (deltas ? 16 : 0);
    key.ptrs[0] = bs.paths.pathBuf.ptr;
    key.ptrs[1] = bs.paths.shadowBuf.ptr;
    key.ptrs[2] = bs.scenes.ptr;
    key.ptrs[3] = bs.chunks.ptr;
    key.ptrs[4] = bs.waves.ptr;
    key.ptrs[5] = bs.paths.queues.ptr;
    key.ptrs[6] = bs.paths.classQueues.ptr;
    bool built = false;
    if (!hostLoop && (!bs.exec || !(bs.key == key))) {
        PRB_CUDA(cudaStreamSynchronize(st));
        build_batch_graph(ds, bs, key);
        built = true;
    }
    const int nWaves = int(waves.size());
    const int maxIter = int(std::min<int64_t>(int64_t(nWaves) * 4200 + 16, int64_t(1) << 30));
    const int halfSlots = capacity / 2;
    float ms = 0.f;
    int64_t launches = 0;
    BatchCtl hc{};
    unsigned long long hs[kStatSlots] = {};
    if (nWaves > 0) {
        k_batch_init<<<1, 32, 0, st>>>(bs.ctl.as<BatchCtl>(), nWaves, maxIter, halfSlots, bs.paths.counters.as<int>(),
                                       bs.paths.stats.as<unsigned long long>());
        PRB_CUDA(cudaEventRecord(bs.ev[0], st));
        if (!hostLoop) {
            PRB_CUDA(cudaGraphLaunch(bs.exec, st));
        } else {
            // Host-driven mode (tools that cannot see inside conditional graphs, e.g. profilers):
            // the same iteration launched directly, the host reading the loop state each time.
            const BatchLaunch L = batch_launch(ds, key);
            BatchCtl *hctl = nullptr;
            PRB_CUDA(cudaMallocHost(&hctl, sizeof(BatchCtl)));
            int iters = 0;
            int perIter = 0;
            for (;;) {
                perIter = enqueue_batch_iteration(st, bs, L, 0, false);
                ++iters;
                PRB_CUDA(cudaMemcpyAsync(hctl, bs.ctl.ptr, sizeof(BatchCtl), cudaMemcpyDeviceToHost, st));
                PRB_CUDA(cudaStreamSynchronize(st));
                if (hctl->filmWave >= hctl->nWaves || (hctl->status & 1) || iters >= maxIter) break;
            }
            cudaFreeHost(hctl);
            bs.launchesPerIteration = perIter;
        }
        PRB_CUDA(cudaEventRecord(bs.ev[1], st));
        PRB_CUDA(cudaMemcpyAsync(&hc, bs.ctl.ptr, sizeof(hc), cudaMemcpyDeviceToHost, st));
        PRB_CUDA(cudaMemcpyAsync(hs, bs.paths.stats.ptr, sizeof(hs), cudaMemcpyDeviceToHost, st));
        PRB_CUDA(cudaStreamSynchronize(st));
        PRB_CUDA(cudaGetLastError());
        PRB_CUDA(cudaEventElapsedTime(&ms, bs.ev[0], bs.ev[1]));
        launches = 1 + int64_t(hc.iter) * bs.launchesPerIteration;
        count_launch(uint64_t(launches));
    }
    int status = 0;
    PRB_CUDA(cudaMemcpy(&status, bs.paths.counters.as<int>() + kCntStatus, sizeof(int), cudaMemcpyDeviceToHost));
    if (hc.status & 1) {
        *err = "batch loop reached its iteration bound";
        return false;
    }
    if (status & kStatusStack) {
        *err = "BVH deeper than the traversal stack (64 entries)";
        return false;
    }
    if (!trial) {
        for (int i = 0; i < count; ++i)
            PRB_CUDA(cudaMemcpyAsync(items[i].outXYZ, films + filmOff[size_t(i)],
                                     size_t(npix[size_t(i)]) * 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
        PRB_CUDA(cudaStreamSynchronize(st));
    }
    if (stats) {
        uint64_t samples = 0;
        for (int i = 0; i < count; ++i) samples += uint64_t(npix[size_t(i)]) * uint64_t(spp[size_t(i)]);
        stats->pathSamples = samples;
        stats->closestRays = hs[kStatClosest];
        stats->shadowRays = hs[kStatShadow];
        stats->waves = uint64_t(nWaves);
        stats->loopIterations = uint64_t(hc.iter);
        stats->deviceMs = ms;
        double wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tHost0).count();
        stats->hostMs = std::max(0.0, wall - ms);
        stats->wavefrontPaths = capacity;
        stats->shadeBlock = shadeBlock;
        stats->graphBuilt = built ? 1 : 0;
    }
    return true;
}

bool check_batch(int count, const prgpu::BatchItem *items, bool needFilms, std::string *err) {
    if (count < 1 || count > kMaxBatch) {
        *err = "batch size must be 1.." + std::to_string(kMaxBatch);
        return false;
    }
    if (!items) {
        *err = "null batch items";
        return false;
    }
    for (int i = 0; i < count; ++i) {
        const prgpu::BatchItem &it = items[i];
        std::string at = "batch item " + std::to_string(i) + ": ";
        if (!it.scene || it.scene->apiVersion != prgpu::kApiVersion) {
            *err = at + "API version mismatch";
            return false;
        }
        if (it.params.spp < 0 || it.params.firstSample < 0) {
            *err = at + "bad render parameters";
            return false;
        }
        if (it.ext && it.ext->structSize != sizeof(prgpu::SceneExt)) {
            *err = at + "SceneExt size mismatch";
            return false;
        }
        if (needFilms && !it.outXYZ) {
            *err = at + "null output film";
            return false;
        }
    }
    return true;
}

// The autotuner: candidate capacities x shading block sizes, each timed (best of two runs after a
// warm-up run that builds its graph) on the batch with every render's spp divided so the trial
// traces about 2^24 path samples.
std::pair<int, int> autotune(DeviceState &ds, BatchState &bs, int count, const prgpu::BatchItem *items,
                             std::string *err, bool *ok) {
    *ok = false;
    uint64_t total = 0;
    for (int i = 0; i < count; ++i)
        total += uint64_t(items[i].scene->camera.width) * items[i].scene->camera.height * uint64_t(items[i].params.spp);
    int div = int(std::max<uint64_t>(1, total / (uint64_t(1) << 24)));
    size_t freeB = 0, totalB = 0;
    PRB_CUDA(cudaMemGetInfo(&freeB, &totalB));
    const int caps[] = {1 << 20, 1 << 21, 1 << 22, 1 << 23};
    const int blocks[] = {128, 256};
    double best = 1e300;
    std::pair<int, int> choice{1 << 22, 256};
    for (int cap : caps) {
        if (size_t(cap) * 512 > freeB / 2) continue;
        for (int sb : blocks) {
            double t = 1e300;
            for (int rep = 0; rep < 3; ++rep) {
                prgpu::BatchStats s{};
                if (!run_batch(ds, bs, count, items, cap, sb, false, true, div, &s, err)) return choice;
                if (rep > 0 && s.pathSamples > 0) t = std::min(t, s.deviceMs / double(s.pathSamples));
            }
            if (t < best) {
                best = t;
                choice = {cap, sb};
            }
        }
    }
    *ok = true;
    return choice;
}

int batch_common(int deviceIndex, int32_t count, const prgpu::BatchItem *items, const prgpu::BatchConfig *config,
                 prgpu::BatchConfig *tuneOut, prgpu::BatchStats *stats, char *err, int errLen) {
    std::lock_guard<std::mutex> lock(gApiMutex);
    try {
        std::string e;
        if (!check_batch(count, items, tuneOut == nullptr, &e)) {
            set_err(err, errLen, e);
            return 1;
        }
        if (config && config->structSize != sizeof(prgpu::BatchConfig)) {
            set_err(err, errLen, "BatchConfig size mismatch");
            return 1;
        }
        if (config && (config->flags & ~1)) {
            set_err(err, errLen, "unknown BatchConfig flags");
            return 1;
        }
        int cap = config ? config->wavefrontPaths : 0, sb = config ? config->shadeBlock : 0;
        if (cap != 0 && (cap < 1024 || cap > (1 << 24))) {
            set_err(err, errLen, "wavefrontPaths out of range (1024 .. 2^24)");
            return 1;
        }
        if (sb != 0 && (sb < 64 || sb > 256 || sb % 64 != 0)) {
            set_err(err, errLen, "shadeBlock must be 64, 128, 192 or 256");
            return 1;
        }
        if (deviceIndex < 0 || deviceIndex >= 64) {
            set_err(err, errLen, "no such GPU device");
            return 1;
        }
        DeviceState &ds = device_state(deviceIndex);
        BatchState &bs = batch_state(deviceIndex);
        bool tunedNow = false;
        if (tuneOut || cap == 0 || sb == 0) {
            uint64_t shape = batch_shape_key(deviceIndex, count, items);
            auto it = bs.tuned.find(shape);
            if (it == bs.tuned.end() || tuneOut) {
                bool ok = false;
                auto c = autotune(ds, bs, count, items, &e, &ok);
                if (!ok) {
                    set_err(err, errLen, e);
                    return 1;
                }
                it = bs.tuned.insert_or_assign(shape, c).first;
                tunedNow = true;
            }
            if (cap == 0) cap = it->second.first;
            if (sb == 0) sb = it->second.second;
            if (tuneOut) {
                tuneOut->structSize = sizeof(prgpu::BatchConfig);
                tuneOut->wavefrontPaths = it->second.first;
                tuneOut->shadeBlock = it->second.second;
                tuneOut->flags = 0;
                return 0;
            }
        }
        if (stats) *stats = prgpu::BatchStats{};
        if (!run_batch(ds, bs, count, items, cap, sb, config && (config->flags & 1), false, 1, stats, &e)) {
            set_err(err, errLen, e);
            return 1;
        }
        if (stats) stats->tuned = tunedNow ? 1 : 0;
        return 0;
    } catch (const CudaError &ex) {
        set_err(err, errLen, ex.msg);
        return 1;
    } catch (const std::exception &ex) {
        set_err(err, errLen, ex.what());
        return 1;
    }
}

} // namespace prb

using namespace prb;

PRGPU_API int prgpu_render(int deviceIndex, const prgpu::SceneDesc *scene, const prgpu::RenderParams *params,
                           float *outXYZ, char *err, int errLen) {
    if (!outXYZ) {
        set_err(err, errLen, "null output film");
        return 1;
    }
    return render_common(deviceIndex, scene, nullptr, params, outXYZ, nullptr, nullptr, err, errLen);
}

PRGPU_API int prgpu_render_ex(int deviceIndex, const prgpu::SceneDesc *scene, const prgpu::SceneExt *ext,
                              const prgpu::RenderParams *params, double *outXYZ, prgpu::RenderStats *stats, char *err,
                              int errLen) {
    if (!outXYZ) {
        set_err(err, errLen, "null output film");
        return 1;
    }
    return render_common(deviceIndex, scene, ext, params, nullptr, outXYZ, stats, err, errLen);
}

PRGPU_API int prgpu_render_aov(int deviceIndex, const prgpu::SceneDesc *sd, const prgpu::SceneExt *ext,
                               const prgpu::AovParams *p, float *outRGB, char *err, int errLen) {
    std::lock_guard<std::mutex> lock(gApiMutex);
    try {
        if (!sd || sd->apiVersion != prgpu::kApiVersion) {
            set_err(err, errLen, "API version mismatch");
            return 1;
        }
        if (!p || !outRGB || p->type < 0 || p->type > 3 || p->spp <= 0 || p->spp > (1 << 20)) {
            set_err(err, errLen, "bad AOV parameters");
            return 1;
        }
        if (p->type == 0 && (p->d65Spectrum < 0 || p->d65Spectrum >= sd->spectrumCount)) {
            set_err(err, errLen, "D65 spectrum index out of range");
            return 1;
        }
        if (ext && ext->structSize != sizeof(prgpu::SceneExt)) {
            set_err(err, errLen, "SceneExt size mismatch");
            return 1;
        }
        if (deviceIndex < 0 || deviceIndex >= 64) {
            set_err(err, errLen, "no such GPU device");
            return 1;
        }
        DeviceState &ds = device_state(deviceIndex);
        RenderState &rs = render_state(deviceIndex);
        std::string e;
        if (!upload_scene(ds, sd, ext, rs.scene, &e)) {
            set_err(err, errLen, e);
            return 1;
        }
        cudaStream_t st = ds.stream;
        const DevScene &scene = rs.scene.ds;
        const size_t n = size_t(sd->camera.width) * size_t(sd->camera.height) * 3;
        rs.sceneTable.ensure(sizeof(DevScene));
        PRB_CUDA(cudaMemcpyAsync(rs.sceneTable.ptr, &scene, sizeof(DevScene), cudaMemcpyHostToDevice, st));
        DevBuf out;
        out.ensure(n * sizeof(float));
        rs.counters.ensure(kCntSlots * sizeof(int));
        int *cnt = rs.counters.as<int>();
        PRB_CUDA(cudaMemsetAsync(cnt, 0, kCntSlots * sizeof(int), st));
        AovArgs a{};
        a.type = p->type;
        a.spp = p->spp;
        a.seed = p->seed;
        a.throughSpecular = p->throughSpecular;
        a.d65 = p->d65Spectrum;
        std::memcpy(a.adapt, p->whiteAdaptation, sizeof(a.adapt));
        std::memcpy(a.toRGB, p->xyzToRGB, sizeof(a.toRGB));
        k_aov<<<ds.prop.multiProcessorCount * 8, 128, 0, st>>>(rs.sceneTable.as<DevScene>(), a, out.as<float>(),
                                                               cnt + kCntStatus);
        count_launch(1);
        PRB_CUDA(cudaGetLastError());
        int status = 0;
        PRB_CUDA(cudaMemcpyAsync(outRGB, out.ptr, n * sizeof(float), cudaMemcpyDeviceToHost, st));
        PRB_CUDA(cudaMemcpyAsync(&status, cnt + kCntStatus, sizeof(int), cudaMemcpyDeviceToHost, st));
        PRB_CUDA(cudaStreamSynchronize(st));
        out.release();
        if (status & kStatusStack) {
            set_err(err, errLen, "traversal stack overflow (BVH deeper than the traversal stack)");
            return 1;
        }
        return 0;
    } catch (const CudaError &ce) {
        set_err(err, errLen, ce.msg);
        return 1;
    }
}

PRGPU_API int prgpu_render_batch(int deviceIndex, int32_t count, const prgpu::BatchItem *items,
                                 const prgpu::BatchConfig *config, prgpu::BatchStats *stats, char *err, int errLen) {
    return batch_common(deviceIndex, count, items, config, nullptr, stats, err, errLen);
}

PRGPU_API int prgpu_autotune_batch(int deviceIndex, int32_t count, const prgpu::BatchItem *items,
                                   prgpu::BatchConfig *out, char *err, int errLen) {
    if (!out) {
        set_err(err, errLen, "null output config");
        return 1;
    }
    return batch_common(deviceIndex, count, items, nullptr, out, nullptr, err, errLen);
}
