// prgpu_trace_rays_noalloc: the ray-query service without any device allocation.
//
// Who needs it: a host that cannot call cudaMalloc / cudaFree while it renders -- for example one
// whose device memory is entirely owned by another allocator's pool (a framework that reserves
// the free HBM for itself), or one that must not trigger the implicit device-wide
// synchronisation that cudaMalloc and cudaFree perform in the middle of its own GPU work.
// prgpu_trace_rays allocates its device copies of the BVH, the rays and the hits on every call;
// this entry point does the same work with every device byte taken from one fixed array that the
// library reserves when it is loaded.
//
// The array g_noalloc_scratch (32 MiB, below) is a file-scope __device__ variable: every GPU on
// which the library's kernels are loaded holds it until the process exits. Its host-side name is
// only a stand-in, so its device address is looked up with cudaGetSymbolAddress once per device,
// on that device's first call. That first call may do more one-time work of the CUDA runtime and
// driver: load this file's kernels (lazy module loading), create the calling thread's per-thread
// default stream, and grow the device's per-thread local-memory reserve for the traversal stack.
// So make one call per device at set-up, before any stream capture and before the point from
// which nothing may allocate; later calls allocate nothing. All calls share the array and it
// keeps the previous call's contents; the status word is cleared at the start of each call. Calls
// that overlapped on the GPU would race on the array, so each call holds the library's lock and
// waits for its own GPU work before it returns: calls made through this entry point run one after
// another. The work is issued on the calling thread's per-thread default stream
// (cudaStreamPerThread), which does not wait for the caller's other streams.
//
// Limits: at most kNoAllocMaxPrims triangles (and 2 * kNoAllocMaxPrims - 1 nodes) per call; any
// number of rays (they stream through a 2^18-ray staging area). The traversal reads the caller's
// node layout directly (no conversion buffers), following pr::BVH::Intersect / IntersectP
// (src/geometry/bvh.cpp:137-232) operation for operation, so its answers are those of
// prgpu_trace_rays and of the reference, bit for bit.

#include <algorithm>

#include "device.cuh"
#include "traverse.cuh"

namespace prb {

constexpr int32_t kNoAllocMaxPrims = 1 << 17;               // 131,072 triangles
constexpr int32_t kNoAllocMaxNodes = 2 * kNoAllocMaxPrims - 1;
constexpr int64_t kNoAllocChunkRays = int64_t(1) << 18;     // rays staged per pass
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;   // 32 MiB

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffStatus = 0;
constexpr size_t kOffNodes = 256;
constexpr size_t kOffOrder = kOffNodes + align256(size_t(kNoAllocMaxNodes) * sizeof(prgpu::BVHNode));
constexpr size_t kOffVerts = kOffOrder + align256(size_t(kNoAllocMaxPrims) * sizeof(int32_t));
constexpr size_t kOffRays = kOffVerts + align256(size_t(kNoAllocMaxPrims) * 9 * sizeof(float));
constexpr size_t kOffPrim = kOffRays + align256(size_t(kNoAllocChunkRays) * sizeof(prgpu::Ray));
constexpr size_t kOffT = kOffPrim + align256(size_t(kNoAllocChunkRays) * sizeof(int32_t));
constexpr size_t kOffB1 = kOffT + align256(size_t(kNoAllocChunkRays) * sizeof(float));
constexpr size_t kOffB2 = kOffB1 + align256(size_t(kNoAllocChunkRays) * sizeof(float));
constexpr size_t kOffEnd = kOffB2 + align256(size_t(kNoAllocChunkRays) * sizeof(float));
static_assert(kOffEnd <= kNoAllocScratchBytes, "no-alloc scratch layout exceeds the array");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Reference-layout traversal: the node's own box is tested when it is visited (bvh.cpp:158-198).
template <bool kAny>
__global__ void __launch_bounds__(256) k_trace_v4(const prgpu::BVHNode *__restrict__ nodes, int32_t nodeCount,
                                                  const int32_t *__restrict__ order, const float *__restrict__ verts,
                                                  const float4 *__restrict__ rays, int64_t n, int32_t *__restrict__ prim,
                                                  float *__restrict__ tOut, float *__restrict__ b1Out,
                                                  float *__restrict__ b2Out, int *__restrict__ status) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        float4 ra = rays[2 * i], rb = rays[2 * i + 1];
        TraceRay r = make_trace_ray(mk(ra.x, ra.y, ra.z), mk(rb.x, rb.y, rb.z));
        float tMax = ra.w;
        int stack[kStackSize];
        int sp = 0, cur = 0, best = -1;
        float bestT = 0.f, bestU = 0.f, bestV = 0.f;
        bool found = false, done = nodeCount == 0;
        while (!done) {
            const prgpu::BVHNode &nd = nodes[cur];
            float tEntry;
            bool boxHit = box_entry(r, nd.bmin.x, nd.bmin.y, nd.bmin.z, nd.bmax.x, nd.bmax.y, nd.bmax.z, &tEntry) &&
                          tEntry < tMax;
            if (boxHit && nd.nPrims == 0) {
                if (sp >= kStackSize) {
                    atomicOr(status, 1);
                    break;
                }
                if (r.neg[nd.axis]) {
                    stack[sp++] = cur + 1;
                    cur = nd.offset;
                } else {
                    stack[sp++] = nd.offset;
                    cur = cur + 1;
                }
                continue;
            }
            if (boxHit) {
                for (int k = 0; k < nd.nPrims; ++k) {
                    int pi = order[nd.offset + k];
                    const float *v = verts + 9 * size_t(pi);
                    float4 v0 = make_float4(v[0], v[1], v[2], 0.f);
                    float4 v1 = make_float4(__fsub_rn(v[3], v[0]), __fsub_rn(v[4], v[1]), __fsub_rn(v[5], v[2]), 0.f);
                    float4 v2 = make_float4(__fsub_rn(v[6], v[0]), __fsub_rn(v[7], v[1]), __fsub_rn(v[8], v[2]), 0.f);
                    float t, u, w;
                    if (hit_triangle(r, v0, v1, v2, tMax, &t, &u, &w)) {
                        found = true;
                        if (kAny) break;
                        tMax = t;
                        best = pi;
                        bestT = t;
                        bestU = u;
                        bestV = w;
                    }
                }
                if (kAny && found) break;
            }
            if (sp == 0) break;
            cur = stack[--sp];
        }
        if (kAny) {
            prim[i] = found ? 1 : 0;
        } else {
            prim[i] = found ? best : -1;
            if (tOut) tOut[i] = found ? bestT : 0.f;
            if (b1Out) b1Out[i] = found ? bestU : 0.f;
            if (b2Out) b2Out[i] = found ? bestV : 0.f;
        }
    }
}

namespace {

unsigned char *gScratchBase[64] = {};

// Checks the caller's tree without allocating: depth-first children after their parent, leaf
// ranges and permutation entries inside the primitive range.
bool validate_v4(const prgpu::BVHNode *nodes, int32_t nodeCount, const int32_t *order, int32_t primCount,
                 std::string *err) {
    for (int32_t i = 0; i < nodeCount; ++i) {
        const prgpu::BVHNode &n = nodes[i];
        if (n.nPrims == 0) {
            if (i + 1 >= nodeCount || n.offset <= i || n.offset >= nodeCount || n.axis > 2) {
                *err = "malformed BVH interior node " + std::to_string(i);
                return false;
            }
        } else if (n.offset < 0 || int64_t(n.offset) + n.nPrims > primCount) {
            *err = "BVH leaf " + std::to_string(i) + " exceeds the primitive range";
            return false;
        }
    }
    for (int32_t s = 0; s < primCount; ++s)
        if (order[s] < 0 || order[s] >= primCount) {
            *err = "primOrder entry out of range";
            return false;
        }
    return true;
}

} // namespace
} // namespace prb

using namespace prb;

PRGPU_API int prgpu_trace_rays_noalloc(int deviceIndex, const prgpu::BVHNode *nodes, int32_t nodeCount,
                                       const int32_t *primOrder, const prgpu::Float3 *triVerts, int32_t primCount,
                                       const prgpu::Ray *rays, int64_t rayCount, int32_t anyHit, int32_t *primOut,
                                       float *tOut, float *b1Out, float *b2Out, char *err, int errLen) {
    std::lock_guard<std::mutex> lock(gApiMutex);
    if (primCount < 0 || nodeCount < 0 || rayCount < 0) {
        set_err(err, errLen, "negative count");
        return 1;
    }
    if (primCount > kNoAllocMaxPrims || nodeCount > kNoAllocMaxNodes) {
        set_err(err, errLen, "prgpu_trace_rays_noalloc handles at most 131072 triangles and 262143 BVH nodes "
                             "per call (its fixed 32 MiB device scratch); use prgpu_trace_rays for larger scenes");
        return 1;
    }
    if ((nodeCount > 0 && !nodes) || (primCount > 0 && (!primOrder || !triVerts)) ||
        (rayCount > 0 && (!rays || !primOut))) {
        set_err(err, errLen, "null argument");
        return 1;
    }
    std::string e;
    if (!validate_v4(nodes, nodeCount, primOrder, primCount, &e)) {
        set_err(err, errLen, e);
        return 1;
    }
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || deviceIndex < 0 || deviceIndex >= devices || deviceIndex >= 64) {
        cudaGetLastError();
        set_err(err, errLen, "no such GPU device");
        return 1;
    }
    try {
        PRB_CUDA(cudaSetDevice(deviceIndex));
        if (!gScratchBase[deviceIndex]) {
            // Once per device, with the device current: the scratch array's device address.
            void *p = nullptr;
            PRB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
            gScratchBase[deviceIndex] = static_cast<unsigned char *>(p);
        }
        unsigned char *base = gScratchBase[deviceIndex];
        int *dStatus = reinterpret_cast<int *>(base + kOffStatus);
        auto *dNodes = reinterpret_cast<prgpu::BVHNode *>(base + kOffNodes);
        auto *dOrder = reinterpret_cast<int32_t *>(base + kOffOrder);
        auto *dVerts = reinterpret_cast<float *>(base + kOffVerts);
        auto *dRays = reinterpret_cast<prgpu::Ray *>(base + kOffRays);
        auto *dPrim = reinterpret_cast<int32_t *>(base + kOffPrim);
        auto *dT = reinterpret_cast<float *>(base + kOffT);
        auto *dB1 = reinterpret_cast<float *>(base + kOffB1);
        auto *dB2 = reinterpret_cast<float *>(base + kOffB2);
        // The per-thread default stream: no stream object to create or destroy, and unlike the
        // legacy stream 0 it does not serialise with the caller's other (blocking) streams.
        cudaStream_t s = cudaStreamPerThread;
        PRB_CUDA(cudaMemsetAsync(dStatus, 0, sizeof(int), s));
        if (nodeCount)
            PRB_CUDA(cudaMemcpyAsync(dNodes, nodes, size_t(nodeCount) * sizeof(prgpu::BVHNode), cudaMemcpyHostToDevice, s));
        if (primCount) {
            PRB_CUDA(cudaMemcpyAsync(dOrder, primOrder, size_t(primCount) * sizeof(int32_t), cudaMemcpyHostToDevice, s));
            PRB_CUDA(cudaMemcpyAsync(dVerts, triVerts, size_t(primCount) * 9 * sizeof(float), cudaMemcpyHostToDevice, s));
        }
        int smCount = 0;
        PRB_CUDA(cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount, deviceIndex));
        for (int64_t off = 0; off < rayCount; off += kNoAllocChunkRays) {
            int64_t cnt = std::min(kNoAllocChunkRays, rayCount - off);
            PRB_CUDA(cudaMemcpyAsync(dRays, rays + off, size_t(cnt) * sizeof(prgpu::Ray), cudaMemcpyHostToDevice, s));
            int grid = int(std::min<int64_t>((cnt + 255) / 256, int64_t(smCount) * 32));
            const auto *r4 = reinterpret_cast<const float4 *>(dRays);
            if (anyHit)
                k_trace_v4<true><<<grid, 256, 0, s>>>(dNodes, nodeCount, dOrder, dVerts, r4, cnt, dPrim, nullptr, nullptr,
                                                      nullptr, dStatus);
            else
                k_trace_v4<false><<<grid, 256, 0, s>>>(dNodes, nodeCount, dOrder, dVerts, r4, cnt, dPrim,
                                                       tOut ? dT : nullptr, b1Out ? dB1 : nullptr,
                                                       b2Out ? dB2 : nullptr, dStatus);
            count_launch();
            PRB_CUDA(cudaGetLastError());
            PRB_CUDA(cudaMemcpyAsync(primOut + off, dPrim, size_t(cnt) * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            if (!anyHit && tOut)
                PRB_CUDA(cudaMemcpyAsync(tOut + off, dT, size_t(cnt) * sizeof(float), cudaMemcpyDeviceToHost, s));
            if (!anyHit && b1Out)
                PRB_CUDA(cudaMemcpyAsync(b1Out + off, dB1, size_t(cnt) * sizeof(float), cudaMemcpyDeviceToHost, s));
            if (!anyHit && b2Out)
                PRB_CUDA(cudaMemcpyAsync(b2Out + off, dB2, size_t(cnt) * sizeof(float), cudaMemcpyDeviceToHost, s));
        }
        int status = 0;
        PRB_CUDA(cudaMemcpyAsync(&status, dStatus, sizeof(int), cudaMemcpyDeviceToHost, s));
        PRB_CUDA(cudaStreamSynchronize(s));
        if (status & 1) {
            set_err(err, errLen, "BVH deeper than the traversal stack (64 entries)");
            return 1;
        }
        return 0;
    } catch (const CudaError &ex) {
        set_err(err, errLen, ex.msg);
        return 1;
    }
}
