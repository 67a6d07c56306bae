// Wavefront spectral volumetric path tracer, single-scene driver (prgpu_render / prgpu_render_ex /
// prgpu_render_aov): one scene per call, the host polling the active-queue length once every few
// bounces. The batched driver (many scenes in one graph launch) is batch.cu.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>
#include <memory>

#include "driver.cuh"
#include "aov.cuh"

namespace prb {
// ---------------------------------------------------------------------------------------------
// Driver

__global__ void __launch_bounds__(256) k_guide_collect(Paths P, float4 *rec, int total, GuideTrainRec *out,
                                                       int *count, int cap) {
    const int span = collect_span(total);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < span; t += gridDim.x * blockDim.x) {
        const int j = collect_path(t, total);
        if (j < total) guide_collect_path(P, rec, j, out, count, cap);
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

std::unique_ptr<RenderState> gRender[64];

void ensure_guide_buffers(RenderState &rs, cudaStream_t st) {
    if (rs.guideCap >= rs.capacity) return;
    rs.guideFeat.ensure(size_t(rs.capacity) * kGuideIn * sizeof(__half));
    rs.guideOut.ensure(size_t(rs.capacity) * kGuideOut * sizeof(float));
    const size_t recBytes = size_t(rs.capacity) * kGuideVertices * 4 * sizeof(float4);
    rs.guideRec.ensure(recBytes);
    PRB_CUDA(cudaMemsetAsync(rs.guideRec.ptr, 0, recBytes, st));
    rs.guideTrain.ensure(size_t(kGuideRecords) * sizeof(GuideTrainRec) + 256);
    rs.guideCap = rs.capacity;
}
GuideTrainRec *guide_train_recs(RenderState &rs) { return rs.guideTrain.as<GuideTrainRec>(); }
int *guide_train_count(RenderState &rs) {
    return reinterpret_cast<int *>(rs.guideTrain.as<unsigned char>() + size_t(kGuideRecords) * sizeof(GuideTrainRec));
}

static size_t carve(char *&p, size_t bytes) {
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

int grid_for(const DeviceState &ds, int64_t work, int perSm) {
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
        ensure_guide_buffers(rs, st);
        trainRecs = guide_train_recs(rs);
        trainCount = guide_train_count(rs);
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
                    k_classify<false><<<gShade, 256, 0, st>>>(scene, nullptr, rs.P, cnt, qin, cq, rs.capacity, guideMode);
                    if (guideMode & 1) {
                        k_guide_features<<<gShade, 256, 0, st>>>(scene, nullptr, rs.P, cnt, cq, rs.capacity,
                                                                 rs.guideFeat.as<__half>(), gopts.bands);
                        guide_infer_rows(st, ds.device, rs.guideFeat.as<__half>(), cnt + kCntClass0 + kClassGuided,
                                         rs.capacity, rs.guideOut.as<float>());
                        launches += 1 + kGuideInferLaunches;
                    }
                    if (timing) PRB_CUDA(cudaEventRecord(rs.ev[4 * b + 1], st));
                    ShadeArgs sa{scene, rs.sceneTable.as<DevScene>(), rs.P, rs.S, cq, rs.capacity, qout, cnt,
                                 rp.maxDepth, 0, rs.guideOut.as<float>(), rs.guideRec.as<float4>(), guideMode, qin,
                                 gopts};
                    const bool dl = scene.deltaCount > 0 || scene.matTex != nullptr;
                    // The plain materials (and training snapshots), then the guided vertices.
                    if (dl) k_shade<false, false, false, true><<<gShade, 256, 0, st>>>(sa);
                    else k_shade<false, false><<<gShade, 256, 0, st>>>(sa);
                    if (guideMode) {
                        if (dl) k_shade<false, true, false, true><<<gShade, 256, 0, st>>>(sa);
                        else k_shade<false, true><<<gShade, 256, 0, st>>>(sa);
                        ++launches;
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

