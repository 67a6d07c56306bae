// Ray-query service (extension entry points prgpu_trace_rays / prgpu_accel_*): closest-hit and
// any-hit traversal of 32-byte rays against a converted caller BVH. One thread per ray over a
// grid sized in multiples of the SM count; rays are read as two 16-byte vector loads and
// results written as coalesced 4-byte stores.

#include <algorithm>
#include <memory>

#include "accel.cuh"

namespace prb {

// Persistent warps: the lanes advance their traversals one node or leaf per iteration, and lanes
// whose ray is done take the next rays from a global counter (one atomic per warp and refill).
// Incoherent rays end after very different numbers of steps; refilling keeps the lanes of a warp
// busy instead of idling until the warp's longest ray ends. A refill (ray load, reciprocal
// direction, root-box test, and the finished rays' result stores) runs once kRefillLanes lanes of
// the warp are idle, or none is busy.

template <bool kAny, bool kWide>
__global__ void __launch_bounds__(256, 4) k_trace_persist(const void *__restrict__ nodes,
                                                          const LeafPrim *__restrict__ prims, RootInfo root,
                                                          const float4 *__restrict__ rays, int64_t n,
                                                          int32_t *__restrict__ primOut, float *__restrict__ tOut,
                                                          float *__restrict__ b1Out, float *__restrict__ b2Out,
                                                          int *__restrict__ status,
                                                          unsigned long long *__restrict__ counter) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int stackRef[kStackSize];
    float stackT[kStackSize];
    // The 4-wide traversal keeps the bottom of its stack in shared memory.
    __shared__ int2 shortStack[kShortStack * 256];
    HybridStack<kShortStack, 256> hs;
    hs.sh = shortStack + threadIdx.x;
    TraceRay r;
    TravState s;
    s.ref = 0;
    s.sp = 0;
    s.tMax = 0.f;
    s.found = false;
    s.hit.prim = -1;
    int64_t idx = 0;
    // pending: this lane's last ray is finished and its result not yet stored.
    bool active = false, exhausted = false, pending = false, overflow = false;
    auto store = [&]() {
        if (kAny) {
            primOut[idx] = s.found ? 1 : 0;
        } else if (kWide) {
            const Hit h = finish_hit<false>(prims, r, s);
            primOut[idx] = h.prim;
            if (tOut) tOut[idx] = h.t;
            if (b1Out) b1Out[idx] = h.u;
            if (b2Out) b2Out[idx] = h.v;
        } else {
            primOut[idx] = s.found ? s.hit.prim : -1;
            if (tOut) tOut[idx] = s.found ? s.hit.t : 0.f;
            if (b1Out) b1Out[idx] = s.found ? s.hit.u : 0.f;
            if (b2Out) b2Out[idx] = s.found ? s.hit.v : 0.f;
        }
    };
    while (true) {
        const bool idle = !active && !exhausted;
        const unsigned need = __ballot_sync(full, idle), busy = __ballot_sync(full, active);
        if (need && (__popc(need) >= kRefillLanes || !busy)) {
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(counter, (unsigned long long)__popc(need));
            base = __shfl_sync(full, base, 0);
            if (idle) {
                if (pending) store();
                idx = int64_t(base) + __popc(need & ((1u << lane) - 1u));
                if (idx >= n) {
                    exhausted = true;
                    pending = false;
                } else {
                    float4 a = __ldcs(rays + 2 * idx), b = __ldcs(rays + 2 * idx + 1);
                    r = make_trace_ray(mk(a.x, a.y, a.z), mk(b.x, b.y, b.z));
                    s.tMax = a.w;
                    s.sp = 0;
                    s.found = false;
                    s.hit.prim = -1;
                    float te;
                    active = !root.empty &&
                             box_entry(r, root.box[0], root.box[1], root.box[2], root.box[3], root.box[4], root.box[5], &te) &&
                             te < s.tMax;
                    s.ref = root.ref;
                    // A ray that misses the root is done at once: a miss, stored at the next refill.
                    pending = !active;
                }
            }
        }
        if (__all_sync(full, exhausted)) break;
        bool done = false;
        if (active) {
            if (kWide)
                done = traverse4_step_st<kAny, false, false, true>(static_cast<const QNode *>(nodes), prims, r, s, hs,
                                                                   &overflow);
            else
                done = traverse_step<kAny, false>(static_cast<const WNode *>(nodes), prims, r, s, stackRef, stackT,
                                                  &overflow);
        }
        if (done) {
            active = false;
            pending = true;
        }
    }
    if (overflow) atomicOr(status, 1);
}

// Resident blocks per SM of a kernel (cached): the persistent grid is exactly one full wave.
template <typename K> int resident_blocks(K kernel, int block) {
    int n = 0;
    PRB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, block, 0));
    return std::max(1, n);
}

// dStatus points at the accel's 16-byte status block: int status at 0, ray counter at 8.
// wide: the 4-wide tree (fast; hits identical up to the order among exactly equal distances);
// otherwise the binary tree in the reference's visit order (bvh.cpp:184-190).
void launch_trace(const DeviceAccel &acc, const prgpu::Ray *dRays, int64_t n, bool anyHit, int32_t *dPrim,
                  float *dT, float *dB1, float *dB2, int *dStatus, cudaStream_t s, int smCount, bool wide) {
    if (n <= 0) return;
    const int block = 256;
    static int resident[2][2] = {{0, 0}, {0, 0}};
    if (!resident[0][0]) {
        resident[0][0] = resident_blocks(k_trace_persist<false, false>, block);
        resident[0][1] = resident_blocks(k_trace_persist<false, true>, block);
        resident[1][0] = resident_blocks(k_trace_persist<true, false>, block);
        resident[1][1] = resident_blocks(k_trace_persist<true, true>, block);
    }
    const void *nodes = wide ? acc.qnodes.ptr : acc.nodes.ptr;
    const int residentAny = resident[1][wide ? 1 : 0], residentClosest = resident[0][wide ? 1 : 0];
    auto *counter = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(dStatus) + 8);
    PRB_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s));
    int64_t blocksNeeded = (n + block - 1) / block;
    const auto *r4 = reinterpret_cast<const float4 *>(dRays);
    if (anyHit) {
        int grid = int(std::min<int64_t>(blocksNeeded, int64_t(smCount) * residentAny));
        if (wide)
            k_trace_persist<true, true><<<grid, block, 0, s>>>(nodes, acc.prims.as<LeafPrim>(), acc.root, r4, n, dPrim,
                                                               nullptr, nullptr, nullptr, dStatus, counter);
        else
            k_trace_persist<true, false><<<grid, block, 0, s>>>(nodes, acc.prims.as<LeafPrim>(), acc.root, r4, n, dPrim,
                                                                nullptr, nullptr, nullptr, dStatus, counter);
    } else {
        int grid = int(std::min<int64_t>(blocksNeeded, int64_t(smCount) * residentClosest));
        if (wide)
            k_trace_persist<false, true><<<grid, block, 0, s>>>(nodes, acc.prims.as<LeafPrim>(), acc.root, r4, n, dPrim,
                                                                dT, dB1, dB2, dStatus, counter);
        else
            k_trace_persist<false, false><<<grid, block, 0, s>>>(nodes, acc.prims.as<LeafPrim>(), acc.root, r4, n,
                                                                 dPrim, dT, dB1, dB2, dStatus, counter);
    }
    count_launch();
    PRB_CUDA(cudaGetLastError());
}

} // namespace prb

using namespace prb;

struct prgpu_accel_t {
    DeviceAccel acc;
    int device = -1;
    DevBuf status;
    DevBuf rays, prim, t, b1, b2;  // staging for the host-buffer path
};

namespace {

bool make_accel(int deviceIndex, const prgpu::BVHNode *nodes, int32_t nodeCount, const int32_t *primOrder,
                const prgpu::Float3 *triVerts, int32_t primCount, prgpu_accel_t *a, std::string *err) {
    if (primCount > 0 && !triVerts) {
        *err = "null triangle array";
        return false;
    }
    HostAccel h;
    if (!convert_bvh(nodes, nodeCount, primOrder, primCount, TriangleSoupSource{triVerts}, &h, err)) return false;
    DeviceState &ds = device_state(deviceIndex);
    a->device = ds.device;
    a->acc.upload(h, ds.stream);
    a->status.ensure(16);  // status word at 0, persistent-kernel ray counter at 8
    PRB_CUDA(cudaMemsetAsync(a->status.ptr, 0, 16, ds.stream));
    PRB_CUDA(cudaStreamSynchronize(ds.stream));
    return true;
}

// Host-buffer query: rays are copied in chunks on the copy stream while the previous chunk is
// traced on the compute stream; results are copied back per chunk. The call is bound by the
// host-to-device copy (32 B per ray in, 4-8 B out); chunks of 2^20 rays (32 MiB) keep the copy
// engine busy while a chunk's trace and result copy (well under its copy time) overlap the next
// chunk's copy, and keep the unoverlapped first copy and last trace of a call short.
bool trace_host(prgpu_accel_t *a, const prgpu::Ray *rays, int64_t n, int anyHit, int32_t *primOut, float *tOut,
                float *b1Out, float *b2Out, bool wide, std::string *err) {
    DeviceState &ds = device_state(a->device);
    const int64_t chunk = int64_t(1) << 20;
    int64_t cap = std::min<int64_t>(n, 2 * chunk);
    a->rays.ensure(size_t(std::max<int64_t>(cap, 1)) * sizeof(prgpu::Ray));
    a->prim.ensure(size_t(std::max<int64_t>(cap, 1)) * sizeof(int32_t));
    if (tOut) a->t.ensure(size_t(std::max<int64_t>(cap, 1)) * sizeof(float));
    if (b1Out) a->b1.ensure(size_t(std::max<int64_t>(cap, 1)) * sizeof(float));
    if (b2Out) a->b2.ensure(size_t(std::max<int64_t>(cap, 1)) * sizeof(float));
    PRB_CUDA(cudaMemsetAsync(a->status.ptr, 0, sizeof(int), ds.stream));
    cudaEvent_t copied[2], traced[2];
    for (int k = 0; k < 2; ++k) {
        PRB_CUDA(cudaEventCreateWithFlags(&copied[k], cudaEventDisableTiming));
        PRB_CUDA(cudaEventCreateWithFlags(&traced[k], cudaEventDisableTiming));
    }
    int64_t nChunks = (n + chunk - 1) / chunk;
    for (int64_t c = 0; c < nChunks; ++c) {
        int slot = int(c & 1);
        int64_t off = c * chunk, cnt = std::min(chunk, n - off);
        int64_t base = int64_t(slot) * chunk;
        // The slot's previous results must be back on the host before it is overwritten.
        if (c >= 2) PRB_CUDA(cudaStreamWaitEvent(ds.copy, traced[slot], 0));
        PRB_CUDA(cudaMemcpyAsync(a->rays.as<prgpu::Ray>() + base, rays + off, size_t(cnt) * sizeof(prgpu::Ray),
                                 cudaMemcpyHostToDevice, ds.copy));
        PRB_CUDA(cudaEventRecord(copied[slot], ds.copy));
        PRB_CUDA(cudaStreamWaitEvent(ds.stream, copied[slot], 0));
        launch_trace(a->acc, a->rays.as<prgpu::Ray>() + base, cnt, anyHit != 0, a->prim.as<int32_t>() + base,
                     tOut ? a->t.as<float>() + base : nullptr, b1Out ? a->b1.as<float>() + base : nullptr,
                     b2Out ? a->b2.as<float>() + base : nullptr, a->status.as<int>(), ds.stream,
                     ds.prop.multiProcessorCount, wide);
        PRB_CUDA(cudaMemcpyAsync(primOut + off, a->prim.as<int32_t>() + base, size_t(cnt) * sizeof(int32_t),
                                 cudaMemcpyDeviceToHost, ds.stream));
        if (tOut)
            PRB_CUDA(cudaMemcpyAsync(tOut + off, a->t.as<float>() + base, size_t(cnt) * sizeof(float),
                                     cudaMemcpyDeviceToHost, ds.stream));
        if (b1Out)
            PRB_CUDA(cudaMemcpyAsync(b1Out + off, a->b1.as<float>() + base, size_t(cnt) * sizeof(float),
                                     cudaMemcpyDeviceToHost, ds.stream));
        if (b2Out)
            PRB_CUDA(cudaMemcpyAsync(b2Out + off, a->b2.as<float>() + base, size_t(cnt) * sizeof(float),
                                     cudaMemcpyDeviceToHost, ds.stream));
        PRB_CUDA(cudaEventRecord(traced[slot], ds.stream));
    }
    int status = 0;
    PRB_CUDA(cudaMemcpyAsync(&status, a->status.ptr, sizeof(int), cudaMemcpyDeviceToHost, ds.stream));
    PRB_CUDA(cudaStreamSynchronize(ds.stream));
    PRB_CUDA(cudaStreamSynchronize(ds.copy));
    for (int k = 0; k < 2; ++k) {
        cudaEventDestroy(copied[k]);
        cudaEventDestroy(traced[k]);
    }
    if (status & 1) {
        *err = "BVH deeper than the traversal stack (64 entries)";
        return false;
    }
    return true;
}

} // namespace

PRGPU_API int prgpu_trace_rays(int deviceIndex, const prgpu::BVHNode *nodes, int32_t nodeCount, const int32_t *primOrder,
                               const prgpu::Float3 *triVerts, int32_t primCount, const prgpu::Ray *rays, int64_t rayCount,
                               int32_t anyHit, int32_t *primOut, float *tOut, float *b1Out, float *b2Out, char *err,
                               int errLen) {
    std::lock_guard<std::mutex> lock(gApiMutex);
    try {
        if (rayCount < 0 || (rayCount > 0 && (!rays || !primOut))) {
            set_err(err, errLen, "bad ray arguments");
            return 1;
        }
        prgpu_accel_t a;
        std::string e;
        bool ok = make_accel(deviceIndex, nodes, nodeCount, primOrder, triVerts, primCount, &a, &e) &&
                  trace_host(&a, rays, rayCount, anyHit, primOut, tOut, b1Out, b2Out, false, &e);
        a.acc.release();
        a.status.release();
        a.rays.release();
        a.prim.release();
        a.t.release();
        a.b1.release();
        a.b2.release();
        if (!ok) {
            set_err(err, errLen, e);
            return 1;
        }
        return 0;
    } catch (const CudaError &e) {
        set_err(err, errLen, e.msg);
        return 1;
    } catch (const std::exception &e) {
        set_err(err, errLen, e.what());
        return 1;
    }
}

PRGPU_API int prgpu_accel_create(int deviceIndex, const prgpu::BVHNode *nodes, int32_t nodeCount, const int32_t *primOrder,
                                 const prgpu::Float3 *triVerts, int32_t primCount, prgpu_accel *out, char *err,
                                 int errLen) {
    std::lock_guard<std::mutex> lock(gApiMutex);
    if (!out) {
        set_err(err, errLen, "null output handle");
        return 1;
    }
    *out = nullptr;
    try {
        auto a = std::make_unique<prgpu_accel_t>();
        std::string e;
        if (!make_accel(deviceIndex, nodes, nodeCount, primOrder, triVerts, primCount, a.get(), &e)) {
            set_err(err, errLen, e);
            return 1;
        }
        *out = a.release();
        return 0;
    } catch (const CudaError &e) {
        set_err(err, errLen, e.msg);
        return 1;
    } catch (const std::exception &e) {
        set_err(err, errLen, e.what());
        return 1;
    }
}

PRGPU_API int prgpu_accel_trace(prgpu_accel accel, const prgpu::Ray *deviceRays, int64_t rayCount, int32_t anyHit,
                                int32_t *devicePrimOut, float *deviceTOut, void *stream, char *err, int errLen) {
    if (!accel || rayCount < 0 || (rayCount > 0 && (!deviceRays || !devicePrimOut))) {
        set_err(err, errLen, "bad arguments");
        return 1;
    }
    try {
        DeviceState &ds = device_state(accel->device);
        launch_trace(accel->acc, deviceRays, rayCount, anyHit != 0, devicePrimOut, deviceTOut, nullptr, nullptr,
                     accel->status.as<int>(), static_cast<cudaStream_t>(stream), ds.prop.multiProcessorCount, true);
        return 0;
    } catch (const CudaError &e) {
        set_err(err, errLen, e.msg);
        return 1;
    }
}

// Host-buffer query against a device-resident BVH (the end-to-end path: rays in and results out
// cross the host link inside the call).
PRGPU_API int prgpu_accel_trace_host(prgpu_accel accel, const prgpu::Ray *rays, int64_t rayCount, int32_t anyHit,
                                     int32_t *primOut, float *tOut, char *err, int errLen) {
    std::lock_guard<std::mutex> lock(gApiMutex);
    if (!accel || rayCount < 0 || (rayCount > 0 && (!rays || !primOut))) {
        set_err(err, errLen, "bad arguments");
        return 1;
    }
    try {
        std::string e;
        if (!trace_host(accel, rays, rayCount, anyHit, primOut, tOut, nullptr, nullptr, true, &e)) {
            set_err(err, errLen, e);
            return 1;
        }
        return 0;
    } catch (const CudaError &e) {
        set_err(err, errLen, e.msg);
        return 1;
    }
}

// Reads back and clears the accel's status word (bit 0: a traversal stack overflowed).
PRGPU_API int prgpu_accel_status(prgpu_accel accel) {
    if (!accel) return -1;
    try {
        DeviceState &ds = device_state(accel->device);
        int s = 0;
        PRB_CUDA(cudaStreamSynchronize(ds.stream));
        PRB_CUDA(cudaMemcpy(&s, accel->status.ptr, sizeof(int), cudaMemcpyDeviceToHost));
        PRB_CUDA(cudaMemset(accel->status.ptr, 0, sizeof(int)));
        return s;
    } catch (const CudaError &) {
        return -1;
    }
}

PRGPU_API int64_t prgpu_accel_bytes(prgpu_accel accel) { return accel ? accel->acc.bytes : 0; }

PRGPU_API void prgpu_accel_destroy(prgpu_accel accel) {
    if (!accel) return;
    std::lock_guard<std::mutex> lock(gApiMutex);
    if (accel->device >= 0) cudaSetDevice(accel->device);
    accel->acc.release();
    accel->status.release();
    accel->rays.release();
    accel->prim.release();
    accel->t.release();
    accel->b1.release();
    accel->b2.release();
    delete accel;
}
