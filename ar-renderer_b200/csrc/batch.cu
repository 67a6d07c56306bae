// Wavefront spectral volumetric path tracer, batched driver (prgpu_render_batch /
// prgpu_autotune_batch): many scenes in one wavefront, run by one CUDA graph launch whose
// device-side loop needs no host round trip, with settings from an autotuner.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>
#include <memory>

#include "driver.cuh"

namespace prb {
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

// Guided batches: the training samples of the wave k_batch_film films this iteration (the same
// half_to_film decision on the same state), from the records of its paths; *count was zeroed
// before. No wave filmed: no samples, and the training launches that follow take no step.
__global__ void __launch_bounds__(256) k_batch_guide_collect(Paths P, const BatchCtl *ctl, const int *counters,
                                                             const BatchWave *waves, float4 *rec, GuideTrainRec *out,
                                                             int *count, int cap) {
    const BatchCtl c = *ctl;
    const int h = half_to_film(c, counters);
    if (h < 0) return;
    const int total = waves[c.filmWave].totalPaths, base = h * c.halfSlots, span = collect_span(total);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < span; t += gridDim.x * blockDim.x) {
        const int j = collect_path(t, total);
        if (j < total) guide_collect_path(P, rec, base + j, out, count, cap);
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

// What a captured batch graph bakes in: launch shapes, kernel variants, buffer addresses and, for
// guided batches, the guide's settings and learning rate (kernel arguments of its launches).
struct BatchGraphKey {
    int capacity = 0, shadeBlock = 0, variant = -1;
    const void *ptrs[12] = {};
    GuideOpts guideOpts;
    float guideLr = 0.f;
    bool operator==(const BatchGraphKey &o) const {
        if (capacity != o.capacity || shadeBlock != o.shadeBlock || variant != o.variant) return false;
        for (int i = 0; i < 12; ++i)
            if (ptrs[i] != o.ptrs[i]) return false;
        return guideOpts.maxSelect == o.guideOpts.maxSelect && guideOpts.logKappaMax == o.guideOpts.logKappaMax &&
               guideOpts.selectLoss == o.guideOpts.selectLoss && guideOpts.trainPasses == o.guideOpts.trainPasses &&
               guideOpts.bands == o.guideOpts.bands && guideOpts.weightClamp == o.guideOpts.weightClamp &&
               guideLr == o.guideLr;
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
    int device = 0;
};

std::unique_ptr<BatchState> gBatch[64];

BatchState &batch_state(int device) {
    auto &p = gBatch[device];
    if (!p) {
        p = std::make_unique<BatchState>();
        p->device = device;
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
    void (*shadeGuided)(ShadeArgs);  // the guided class, when the batch uses the guide
    void (*shadeFull)(ShadeArgs);
    bool walls, full;
    int guideMode;  // OR of the renders' guide flags (bit 0 sample, bit 1 train): the guide launches run
    GuideOpts guideOpts;
    int gExtend, gShadow, gShade, gWide, shadeBlock, capacity;
};

BatchLaunch batch_launch(const DeviceState &ds, const BatchGraphKey &key) {
    const bool sph = key.variant & 1, media = key.variant & 2;
    BatchLaunch L{};
    L.walls = key.variant & 4;
    L.full = key.variant & 8;
    const bool dl = key.variant & 16;
    L.guideMode = (key.variant >> 5) & 3;
    L.guideOpts = key.guideOpts;
    L.shade = dl ? k_shade<true, false, false, true> : k_shade<true>;
    L.shadeGuided = dl ? k_shade<true, true, false, true> : k_shade<true, true>;
    L.shadeFull = dl ? k_shade<true, false, true, true> : k_shade<true, false, true>;
    L.extend = sph ? k_extend<true, true> : k_extend<false, true>;
    L.shadowAny = L.walls ? (sph ? k_shadow_any<true, true, true, true> : k_shadow_any<false, true, true, true>)
                  : sph   ? (media ? k_shadow_any<true, true, true> : k_shadow_any<true, false, true>)
                          : (media ? k_shadow_any<false, true, true> : k_shadow_any<false, false, true>);
    L.shadowWalk = sph ? k_shadow_walk<true, true> : k_shadow_walk<false, true>;
    const int sms = ds.prop.multiProcessorCount;
    L.gExtend = sms * resident_blocks_of(L.extend);
    L.gShadow = sms * resident_blocks_of(L.shadowAny);
    // Shading: four waves of resident blocks, not one. The cost per path varies widely (media,
    // next-event estimation, termination), and with a single wave the SMs whose blocks drew the
    // heavy paths finished last while the others idled (12 renders of the uneven batch at 1/8 of
    // their spp: 619 ms with one wave, 578 ms with four, as fast as the same renders one by one).
    int perSm = 0;
    PRB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, L.shade, key.shadeBlock, 0));
    L.gShade = sms * std::max(1, perSm) * 4;
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
    const int device = bs.device;
    for (int b = 0; b < 2; ++b) {
        L.extend<<<L.gExtend, 256, 0, st>>>(none, scenes, rs.P, cnt, qin);
        k_classify<true><<<L.gWide, 256, 0, st>>>(none, scenes, rs.P, cnt, qin, cq, rs.capacity);
        if (L.guideMode & 1) {
            // Network inference for the diffuse class queue (each path's render decides whether its
            // vertex uses the result).
            k_guide_features<true><<<L.gWide, 256, 0, st>>>(none, scenes, rs.P, cnt, cq, rs.capacity,
                                                           rs.guideFeat.as<__half>(), L.guideOpts.bands);
            guide_infer_rows(st, device, rs.guideFeat.as<__half>(), cnt + kCntClass0 + kClassGuided, rs.capacity,
                             rs.guideOut.as<float>());
            launches += 1 + kGuideInferLaunches;
        }
        ShadeArgs sa{none, scenes, rs.P, rs.S, cq, rs.capacity, qout, cnt, 0, L.capacity / 2,
                     L.guideMode ? rs.guideOut.as<float>() : nullptr, L.guideMode ? rs.guideRec.as<float4>() : nullptr,
                     L.guideMode, qin, L.guideOpts};
        L.shade<<<L.gShade, L.shadeBlock, 0, st>>>(sa);
        if (L.guideMode) {
            L.shadeGuided<<<L.gShade, L.shadeBlock, 0, st>>>(sa);
            ++launches;
        }
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
    if (L.guideMode & 2) {
        // Online training on the filmed wave's samples: one Adam step per kGuideBatch samples.
        GuideTrainRec *recs = guide_train_recs(rs);
        int *count = guide_train_count(rs);
        PRB_CUDA(cudaMemsetAsync(count, 0, sizeof(int), st));
        k_batch_guide_collect<<<L.gWide, 256, 0, st>>>(rs.P, ctl, cnt, waves, rs.guideRec.as<float4>(), recs, count,
                                                       kGuideRecords);
        for (int pass = 0; pass < L.guideOpts.trainPasses; ++pass)
            for (int k = 0; k < kGuideRecords / kGuideBatch; ++k)
                guide_train_records(st, device, recs, count, k * kGuideBatch, kGuideBatch, 0.f);
        launches += 1 + L.guideOpts.trainPasses * (kGuideRecords / kGuideBatch) * kGuideTrainLaunches;
    }
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
    // Guided renders: SceneExt::flags of each item (bit 0 sample with the guide, bit 1 train it
    // online, bit 2 fresh weights first); one network serves the whole batch.
    int guideMode = 0;
    bool guideReset = false;
    uint64_t guideSeed = 0;
    for (int i = 0; i < count; ++i) {
        const int f = items[i].ext ? items[i].ext->flags : 0;
        if (f & 3) {
            if (!guideMode) guideSeed = items[i].params.seed;
            guideMode |= f & 3;
            guideReset = guideReset || (f & 4);
        }
    }
    // Autotuning trials sample with the guide but never train it (they must not change its weights).
    if (trial) {
        guideMode &= 1;
        guideReset = false;
    }
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
    if (guideMode) {
        guide_prepare(ds, ds.device, guideReset, guideSeed);
        ensure_guide_buffers(bs.paths, st);
        guide_reserve_training(ds.device, kGuideBatch);
    }
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
        d.guideMode = items[i].ext ? (items[i].ext->flags & guideMode) : 0;
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
    key.variant = sph | (media ? 2 : 0) | (walls ? 4 : 0) | (full ? 8 : 0) | (deltas ? 16 : 0) | (guideMode << 5);
    key.ptrs[0] = bs.paths.pathBuf.ptr;
    key.ptrs[1] = bs.paths.shadowBuf.ptr;
    key.ptrs[2] = bs.scenes.ptr;
    key.ptrs[3] = bs.chunks.ptr;
    key.ptrs[4] = bs.waves.ptr;
    key.ptrs[5] = bs.paths.queues.ptr;
    key.ptrs[6] = bs.paths.classQueues.ptr;
    if (guideMode) {
        key.ptrs[7] = bs.paths.guideFeat.ptr;
        key.ptrs[8] = bs.paths.guideOut.ptr;
        key.ptrs[9] = bs.paths.guideRec.ptr;
        key.ptrs[10] = bs.paths.guideTrain.ptr;
        key.ptrs[11] = guide_training_buffer(ds.device);
        key.guideOpts = guide_options(ds.device);
        key.guideLr = guide_learning_rate(ds.device);
    }
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
