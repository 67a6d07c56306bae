// Path-guiding network on the 5th-generation tensor cores (tcgen05, sm_100a): inference over a
// batch of shading points and one fused training pass (forward, loss gradient, backward, weight
// gradients), FP16 operands from shared memory, FP32 accumulators in tensor memory (TMEM).
// Network and loss: guide.cuh. No counterpart in the reference renderer.
//
// One CTA = 4 warps = 128 rows (shading points / training samples) per tile; persistent CTAs loop
// over tiles. Every GEMM is D[128 x N] (+)= A[128 x K] B[K x N] issued by one thread as K/16
// tcgen05.mma instructions (kind::f16, M = 128), completion signalled through an mbarrier by
// tcgen05.commit; then each warp reads its 32 TMEM lanes (= its 32 rows) with tcgen05.ld.
//
// Shared-memory operand layout ("interleaved", no swizzle): a tile of R rows x K columns of FP16
// is a grid of 8 x 8 core matrices (128 contiguous bytes, one 16-byte row each), row groups
// fastest: element (r, k) at byte ((k / 8) * (R / 8) + r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2.
//   * as a K-major operand (rows = M or N): leading byte offset (between the two 8-column core
//     matrices of one K step of 16) = (R / 8) * 128, stride byte offset (between 8-row groups) = 128;
//   * the transpose of the same tile (rows become K) is an MN-major operand with leading byte
//     offset 128 (between 8-row groups, now K) and stride byte offset (R / 8) * 128 (between
//     8-column groups, now M or N).
// So the backward pass reuses the forward tiles: dH = dZ W reads W^T (MN-major) and dW = dZ^T A
// reads A^T and dZ^T (MN-major), with no transposed copies.
//
// Weight gradients for layers with 64 inputs use M = 128 as well: rows 64..127 of that D read
// the next tile in shared memory and are discarded (rows of D are independent).

#include <cuda_fp16.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "device.cuh"
#include "guide.cuh"
#include "guide_host.h"
#include "../../include/prgpu_api.h"

namespace prb {

constexpr int kTileRows = 128;
constexpr int kWTotalBytes = kGuideParams * 2;  // 47,104
constexpr unsigned kWaitLimit = 1u << 20;       // mbarrier polls before giving up (status bit)

__host__ __device__ constexpr int weight_byte_offset(int l) { return 2 * guide_weight_offset(l); }

__host__ __device__ __forceinline__ int tile_byte(int r, int k, int R) {
    return ((k >> 3) * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t start, uint32_t lbo, uint32_t sbo) {
    return uint64_t((start >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);  // version 1, no swizzle
}

// K-major operand: the tile's rows are M (or N), K step k0 (multiple of 16).
__device__ __forceinline__ uint64_t desc_k(uint32_t base, int R, int k0) {
    return umma_desc(base + (k0 >> 3) * (R >> 3) * 128, (R >> 3) * 128, 128);
}
// MN-major operand: the tile's rows are K (K step k0), its columns M (or N).
__device__ __forceinline__ uint64_t desc_mn(uint32_t base, int R, int k0) {
    return umma_desc(base + (k0 >> 3) * 128, 128, (R >> 3) * 128);
}

__host__ __device__ constexpr uint32_t idesc_f16(int M, int N, int aMN, int bMN) {
    return (1u << 4) | (uint32_t(aMN) << 15) | (uint32_t(bMN) << 16) | (uint32_t(N >> 3) << 17) |
           (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
    uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(dtmem), "l"(a), "l"(b), "r"(idesc), "r"(accum), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Waits for the mbarrier phase `parity` to complete, at most kWaitLimit polls; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (unsigned i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// TMEM allocation by warp 0 (columns: power of two >= 32); the address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                     "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
    if (threadIdx.x < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar) {
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
}

// Copies the packed FP16 weights (already in the interleaved layout) into shared memory.
__device__ __forceinline__ void load_weights(unsigned char *w, const __half *packed) {
    const int4 *src = reinterpret_cast<const int4 *>(packed);
    int4 *dst = reinterpret_cast<int4 *>(w);
    for (int i = threadIdx.x; i < kWTotalBytes / 16; i += blockDim.x) dst[i] = src[i];
}

// One GEMM of the network: issue K/16 MMAs into D (one thread), wait for completion (all).
// aMN / bMN select MN-major operands; descriptors come from the tile bases.
struct Gemm {
    uint32_t d;            // TMEM address of D
    uint32_t a, b;         // smem bases of the A and B tiles
    int aRows, bRows;      // R of the tiles (their row counts)
    int M, N, K;
    int aMN, bMN;
    bool accumulate;       // add onto D (else D = A B)
};

__device__ __forceinline__ bool run_gemm(const Gemm &g, uint32_t mbar, uint32_t &phase) {
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (threadIdx.x == 0) {
        const uint32_t id = idesc_f16(g.M, g.N, g.aMN, g.bMN);
        for (int k0 = 0; k0 < g.K; k0 += 16) {
            uint64_t ad = g.aMN ? desc_mn(g.a, g.aRows, k0) : desc_k(g.a, g.aRows, k0);
            uint64_t bd = g.bMN ? desc_mn(g.b, g.bRows, k0) : desc_k(g.b, g.bRows, k0);
            mma_f16(g.d, ad, bd, id, (g.accumulate || k0 > 0) ? 1u : 0u);
        }
        mma_commit(mbar);
    }
    // Every thread polls the same barrier; the vote keeps the outcome uniform across the CTA, so a
    // timeout cannot split the threads between two barriers.
    bool ok = __syncthreads_and(mbar_wait(mbar, phase)) != 0;
    phase ^= 1u;
    tc_after_sync();
    return ok;
}

__device__ __forceinline__ void put_half(unsigned char *tile, int r, int k, int R, float v) {
    *reinterpret_cast<__half *>(tile + tile_byte(r, k, R)) = __float2half_rn(v);
}

// Writes this thread's row of a hidden activation: ReLU, unit 63 held at 1, FP16.
__device__ __forceinline__ void store_hidden(unsigned char *tile, int r, const float *z) {
#pragma unroll
    for (int k = 0; k < kGuideHid; ++k) put_half(tile, r, k, kTileRows, k == kGuideConstHid ? 1.f : fmaxf(z[k], 0.f));
}

__device__ __forceinline__ void tmem_row(uint32_t tbase, int ncols, float *v) {
    const uint32_t lane = (threadIdx.x >> 5) * 32;
    for (int c = 0; c < ncols; c += 16) tmem_ld16(tbase + (lane << 16) + uint32_t(c), v + c);
}

// ---------------------------------------------------------------------------------------------
// Inference: rows of FP16 features [n x 128] -> FP32 outputs [n x 48]. n is read on the device.

struct GuideSmemFwd {
    unsigned char x[kTileRows * kGuideIn * 2];  // 32 KB input tile
    unsigned char h[kTileRows * kGuideHid * 2]; // 16 KB activation tile (reused by every layer)
    unsigned char w[kWTotalBytes];
    uint64_t bar;
    uint32_t tmem;
};

__global__ void __launch_bounds__(128, 1) k_guide_forward(const __half *__restrict__ features, const int *count,
                                                          const __half *__restrict__ packed, float *out, int *status) {
    extern __shared__ __align__(1024) unsigned char smraw[];
    GuideSmemFwd &S = *reinterpret_cast<GuideSmemFwd *>(smraw);
    const int n = *count;
    const int tiles = (n + kTileRows - 1) / kTileRows;
    if (int(blockIdx.x) >= tiles) return;
    load_weights(S.w, packed);
    mbar_init(&S.bar);
    tmem_alloc(&S.tmem, 64);
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tm = S.tmem, mbar = smem_u32(&S.bar);
    const uint32_t xs = smem_u32(S.x), hs = smem_u32(S.h), ws = smem_u32(S.w);
    uint32_t phase = 0;
    bool ok = true;
    const int r = threadIdx.x;
    float z[kGuideHid];
    for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        const int row = t * kTileRows + r;
        // Input tile: 16-byte groups of 8 features straight into their core-matrix rows.
        const int4 *src = reinterpret_cast<const int4 *>(features + size_t(row) * kGuideIn);
        for (int g = 0; g < kGuideIn / 8; ++g) {
            int4 v = row < n ? src[g] : make_int4(0, 0, 0, 0);
            *reinterpret_cast<int4 *>(S.x + tile_byte(r, 8 * g, kTileRows)) = v;
        }
        for (int l = 0; l < kGuideLayers && ok; ++l) {
            const int K = guide_layer_in(l), N = guide_layer_out(l);
            Gemm g{tm, l == 0 ? xs : hs, ws + uint32_t(weight_byte_offset(l)), kTileRows, N, kTileRows, N, K, 0, 0, false};
            ok = run_gemm(g, mbar, phase);
            if (!ok) break;
            tmem_row(tm, N, z);
            if (l < kGuideLayers - 1) {
                // All MMAs of this layer have completed: the activation tile may be overwritten.
                store_hidden(S.h, r, z);
            } else if (row < n) {
                float4 *o = reinterpret_cast<float4 *>(out + size_t(row) * kGuideOut);
#pragma unroll
                for (int c = 0; c < kGuideOut / 4; ++c) o[c] = make_float4(z[4 * c], z[4 * c + 1], z[4 * c + 2], z[4 * c + 3]);
            }
            tc_before_sync();
            __syncthreads();
            tc_after_sync();
        }
    }
    if (!ok && threadIdx.x == 0) atomicOr(status, 1);
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    tmem_free(tm, 64);
}

// ---------------------------------------------------------------------------------------------
// Training pass: per sample (FP16 features, wi, pb, w) -> summed loss and the gradient of the
// summed loss with respect to every weight (FP32, added into grad). Weight gradients accumulate
// in TMEM over all tiles of a CTA and are added to global memory once per CTA.

struct GuideSample {
    float wi[3];
    float pb;
    float w;
    float n[3];   // shading normal (the folding plane)
};

struct GuideSmemTrain {
    unsigned char x[kTileRows * kGuideIn * 2];            // 32 KB
    unsigned char h[4][kTileRows * kGuideHid * 2];        // 4 x 16 KB (H1..H4)
    unsigned char dz[2][kTileRows * kGuideHid * 2];       // 2 x 16 KB (dZ ping-pong; dz[0] also holds
                                                          // the 48-wide output gradient)
    unsigned char w[kWTotalBytes];
    uint64_t bar;
    uint32_t tmem;
    float loss[4];
};

// TMEM columns: [0, 64) scratch D; then dW accumulators: layer 0 (64 cols), layers 1..3 (64
// each), layer 4 (48) -> 368 of 512.
__host__ __device__ constexpr uint32_t dw_col(int l) { return 64 + 64 * uint32_t(l); }

__global__ void __launch_bounds__(128, 1) k_guide_train(const __half *__restrict__ features,
                                                        const GuideSample *__restrict__ samples, const int *count,
                                                        const __half *__restrict__ packed, float *grad,
                                                        float *lossSum, int *status, const float *wnorm,
                                                        GuideOpts opts) {
    extern __shared__ __align__(1024) unsigned char smraw[];
    GuideSmemTrain &S = *reinterpret_cast<GuideSmemTrain *>(smraw);
    const int n = *count;
    const int tiles = (n + kTileRows - 1) / kTileRows;
    if (int(blockIdx.x) >= tiles) return;
    load_weights(S.w, packed);
    mbar_init(&S.bar);
    tmem_alloc(&S.tmem, 512);
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tm = S.tmem, mbar = smem_u32(&S.bar);
    const uint32_t xs = smem_u32(S.x), ws = smem_u32(S.w);
    uint32_t hs[4], dzs[2];
    for (int i = 0; i < 4; ++i) hs[i] = smem_u32(S.h[i]);
    for (int i = 0; i < 2; ++i) dzs[i] = smem_u32(S.dz[i]);
    uint32_t phase = 0;
    bool ok = true, firstTile = true;
    const int r = threadIdx.x;
    const float wscale = wnorm ? *wnorm : 1.f;
    float z[kGuideHid], lossAcc = 0.f;
    for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        const int row = t * kTileRows + r;
        const bool valid = row < n;
        const int4 *src = reinterpret_cast<const int4 *>(features + size_t(row) * kGuideIn);
        for (int g = 0; g < kGuideIn / 8; ++g) {
            int4 v = valid ? src[g] : make_int4(0, 0, 0, 0);
            *reinterpret_cast<int4 *>(S.x + tile_byte(r, 8 * g, kTileRows)) = v;
        }
        // Forward, keeping H1..H4.
        for (int l = 0; l < kGuideLayers && ok; ++l) {
            const int K = guide_layer_in(l), N = guide_layer_out(l);
            Gemm g{tm, l == 0 ? xs : hs[l - 1], ws + uint32_t(weight_byte_offset(l)), kTileRows, N, kTileRows, N, K,
                   0, 0, false};
            ok = run_gemm(g, mbar, phase);
            if (!ok) break;
            tmem_row(tm, N, z);
            if (l < kGuideLayers - 1) {
                store_hidden(S.h[l], r, z);
            } else {
                // Output gradient of this row (zero for padding rows), FP16 into dz[0] (48 wide).
                float gout[kGuideOut];
                if (valid) {
                    const GuideSample sm = samples[row];
                    // The clamp applies to online batches (weights normalised to mean 1), not to
                    // the caller-weighted gradient of prgpu_guide_gradient.
                    const float wn = (wnorm && opts.weightClamp > 0.f) ? fminf(sm.w * wscale, opts.weightClamp)
                                                                       : sm.w * wscale;
                    lossAcc += guide_loss_grad(z, mk(sm.wi[0], sm.wi[1], sm.wi[2]), mk(sm.n[0], sm.n[1], sm.n[2]),
                                               sm.pb, wn, gout, opts);
                } else {
#pragma unroll
                    for (int k = 0; k < kGuideOut; ++k) gout[k] = 0.f;
                }
#pragma unroll
                for (int k = 0; k < kGuideOut; ++k) put_half(S.dz[0], r, k, kTileRows, gout[k]);
            }
            tc_before_sync();
            __syncthreads();
            tc_after_sync();
        }
        // Backward: layer l's dZ is in dz[cur]; dW_l += A_{l-1}^T dZ_l; dH_{l-1} = dZ_l W_l.
        int cur = 0;
        for (int l = kGuideLayers - 1; l >= 0 && ok; --l) {
            const int K = guide_layer_in(l), N = guide_layer_out(l);
            // dW_l [K x N] += A^T [K x 128] dZ [128 x N]: M = 128 (rows >= K discarded).
            Gemm gw{tm + dw_col(l), l == 0 ? xs : hs[l - 1], dzs[cur], kTileRows, kTileRows, 128, N, kTileRows,
                    1, 1, !firstTile};
            ok = run_gemm(gw, mbar, phase);
            if (!ok || l == 0) break;
            // dH_{l-1} [128 x K] = dZ [128 x N] W_l [N x K]: A K-major (K = N), B = W_l^T MN-major.
            Gemm gd{tm, dzs[cur], ws + uint32_t(weight_byte_offset(l)), kTileRows, N, kTileRows, K, N, 0, 1, false};
            ok = run_gemm(gd, mbar, phase);
            if (!ok) break;
            tmem_row(tm, K, z);
            // dZ_{l-1} = dH * relu'(Z_{l-1}) (from the stored activation), constant unit 0.
            const unsigned char *hprev = S.h[l - 1];
#pragma unroll 8
            for (int k = 0; k < kGuideHid; ++k) {
                float hv = __half2float(*reinterpret_cast<const __half *>(hprev + tile_byte(r, k, kTileRows)));
                float v = (k == kGuideConstHid || !(hv > 0.f)) ? 0.f : z[k];
                put_half(S.dz[cur ^ 1], r, k, kTileRows, v);
            }
            cur ^= 1;
            tc_before_sync();
            __syncthreads();
            tc_after_sync();
        }
        firstTile = false;
    }
    if (!ok && threadIdx.x == 0) atomicOr(status, 1);
    // Per-CTA weight gradients: TMEM lane = input feature (row of dW^T), columns = outputs.
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (ok) {
        for (int l = 0; l < kGuideLayers; ++l) {
            const int K = guide_layer_in(l), N = guide_layer_out(l);
            float v[kGuideHid];
            tmem_row(tm + dw_col(l), N, v);
            if (r < K) {
                float *gl = grad + guide_weight_offset(l);
                for (int c = 0; c < N; ++c)
                    if (v[c] != 0.f) atomicAdd(gl + size_t(c) * K + r, v[c]);
            }
        }
        // Loss: warp sums, one atomic per warp.
        for (int o = 16; o > 0; o >>= 1) lossAcc += __shfl_xor_sync(0xffffffffu, lossAcc, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(lossSum, lossAcc);
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    tmem_free(tm, 512);
}

// ---------------------------------------------------------------------------------------------
// Parameter packing and Adam.

// FP32 master weights -> FP16 in the interleaved layout of each layer's [out x in] tile.
__global__ void k_guide_pack(const float *master, __half *packed) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kGuideParams; i += gridDim.x * blockDim.x) {
        int l = 0;
        while (l + 1 < kGuideLayers && i >= guide_weight_offset(l + 1)) ++l;
        const int local = i - guide_weight_offset(l), K = guide_layer_in(l), R = guide_layer_out(l);
        const int o = local / K, k = local - o * K;
        packed[(weight_byte_offset(l) + tile_byte(o, k, R)) / 2] = __float2half_rn(master[i]);
    }
}

// Adam on the gradient times scale (or *scaleDev: 0 = an empty online batch, no step). The step
// count for the bias correction lives on the device (*stepDev, advanced before this kernel by
// k_guide_norm or k_guide_bump), so captured graphs that replay training stay correct.
__global__ void k_guide_adam(float *master, float *m, float *v, const float *grad, float scale, const float *scaleDev,
                             float lr, float b1, float b2, float eps, const int *stepDev) {
    if (scaleDev) {
        scale = *scaleDev;
        if (scale == 0.f) return;
    }
    const int step = *stepDev;
    const float c1 = 1.f - powf(b1, float(step)), c2 = 1.f - powf(b2, float(step));
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kGuideParams; i += gridDim.x * blockDim.x) {
        float g = grad[i] * scale;
        float mi = b1 * m[i] + (1.f - b1) * g;
        float vi = b2 * v[i] + (1.f - b2) * g * g;
        m[i] = mi;
        v[i] = vi;
        master[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

__global__ void k_guide_bump(int *stepDev) { ++*stepDev; }

__global__ void k_guide_to_half(const float *in, __half *out, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = __float2half_rn(in[i]);
}

// ---------------------------------------------------------------------------------------------
// Host side: per-device guide state and launchers.

struct GuideState {
    DevBuf master, m, v, grad, packed, scratch, loss, status, train;
    DevBuf stepDev;        // Adam steps taken (int, device)
    bool ready = false;
    int sms = 0;
    float lr = 1e-3f;      // online learning rate (Adam)
    GuideOpts opts;        // sampling and training settings
};

GuideState gGuide[64];

size_t fwd_smem() { return sizeof(GuideSmemFwd) + 1024; }
size_t train_smem() { return sizeof(GuideSmemTrain) + 1024; }

void guide_setup(DeviceState &ds, GuideState &g) {
    if (g.ready) return;
    g.master.ensure(kGuideParams * sizeof(float));
    g.m.ensure(kGuideParams * sizeof(float));
    g.v.ensure(kGuideParams * sizeof(float));
    g.grad.ensure(kGuideParams * sizeof(float));
    g.packed.ensure(kWTotalBytes);
    g.loss.ensure(sizeof(float) * 4);
    g.status.ensure(sizeof(int) * 4);
    g.stepDev.ensure(sizeof(int));
    PRB_CUDA(cudaMemsetAsync(g.stepDev.ptr, 0, sizeof(int), ds.stream));
    PRB_CUDA(cudaMemsetAsync(g.master.ptr, 0, kGuideParams * sizeof(float), ds.stream));
    PRB_CUDA(cudaMemsetAsync(g.m.ptr, 0, kGuideParams * sizeof(float), ds.stream));
    PRB_CUDA(cudaMemsetAsync(g.v.ptr, 0, kGuideParams * sizeof(float), ds.stream));
    PRB_CUDA(cudaMemsetAsync(g.status.ptr, 0, sizeof(int) * 4, ds.stream));
    PRB_CUDA(cudaFuncSetAttribute(k_guide_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, int(fwd_smem())));
    PRB_CUDA(cudaFuncSetAttribute(k_guide_train, cudaFuncAttributeMaxDynamicSharedMemorySize, int(train_smem())));
    g.sms = ds.prop.multiProcessorCount;
    g.ready = true;
}

void guide_set_weights(DeviceState &ds, GuideState &g, const float *host) {
    PRB_CUDA(cudaMemcpyAsync(g.master.ptr, host, kGuideParams * sizeof(float), cudaMemcpyHostToDevice, ds.stream));
    PRB_CUDA(cudaMemsetAsync(g.m.ptr, 0, kGuideParams * sizeof(float), ds.stream));
    PRB_CUDA(cudaMemsetAsync(g.v.ptr, 0, kGuideParams * sizeof(float), ds.stream));
    PRB_CUDA(cudaMemsetAsync(g.stepDev.ptr, 0, sizeof(int), ds.stream));
    k_guide_pack<<<64, 256, 0, ds.stream>>>(g.master.as<float>(), g.packed.as<__half>());
    count_launch();
}

// Launches inference over n rows (device count); features FP16 [n x 128], out FP32 [n x 48].
void guide_forward(cudaStream_t st, GuideState &g, const __half *features, const int *dcount, int maxRows, float *out) {
    int tiles = (maxRows + kTileRows - 1) / kTileRows;
    int grid = std::max(1, std::min(tiles, g.sms * 2));
    k_guide_forward<<<grid, 128, fwd_smem(), st>>>(features, dcount, g.packed.as<__half>(), out, g.status.as<int>());
    count_launch();
}

void guide_train(cudaStream_t st, GuideState &g, const __half *features, const GuideSample *samples, const int *dcount,
                 int maxRows) {
    int tiles = (maxRows + kTileRows - 1) / kTileRows;
    int grid = std::max(1, std::min(tiles, g.sms));
    PRB_CUDA(cudaMemsetAsync(g.grad.ptr, 0, kGuideParams * sizeof(float), st));
    PRB_CUDA(cudaMemsetAsync(g.loss.ptr, 0, sizeof(float), st));
    k_guide_train<<<grid, 128, train_smem(), st>>>(features, samples, dcount, g.packed.as<__half>(), g.grad.as<float>(),
                                                   g.loss.as<float>(), g.status.as<int>(), nullptr, g.opts);
    count_launch();
}

void guide_adam(cudaStream_t st, GuideState &g, float scale, float lr) {
    k_guide_bump<<<1, 1, 0, st>>>(g.stepDev.as<int>());
    k_guide_adam<<<64, 256, 0, st>>>(g.master.as<float>(), g.m.as<float>(), g.v.as<float>(), g.grad.as<float>(), scale,
                                     nullptr, lr, 0.9f, 0.999f, 1e-8f, g.stepDev.as<int>());
    k_guide_pack<<<64, 256, 0, st>>>(g.master.as<float>(), g.packed.as<__half>());
    count_launch(3);
}

// Online training: recorded samples -> FP16 features and loss inputs for up to maxRows rows, the
// batch's weight sum, then the normalisation (weights to mean 1) and the Adam scale (1 / rows).
__global__ void k_guide_prep(const GuideTrainRec *recs, const int *count, int offset, int maxRows, __half *features,
                             GuideSample *samples, int *rows, float *wsum, int bands) {
    const int n = max(0, min(*count - offset, maxRows));
    recs += offset;
    if (blockIdx.x == 0 && threadIdx.x == 0) *rows = n;
    // Every thread runs the same number of iterations (whole warps per iteration), so the weight
    // sum is reduced per warp: one atomic per warp instead of one per row on a single address.
    const int stride = gridDim.x * blockDim.x;
    const int iters = (n + stride - 1) / stride;
    for (int it = 0, i = blockIdx.x * blockDim.x + threadIdx.x; it < iters; ++it, i += stride) {
        float w = 0.f;
        if (i < n) {
            const GuideTrainRec r = recs[i];
            float f[kGuideIn];
#pragma unroll
            for (int k = 0; k < kGuideIn; ++k) f[k] = 0.f;
            guide_features_n(r.xn, mk(r.n[0], r.n[1], r.n[2]), mk(r.wo[0], r.wo[1], r.wo[2]), f, bands);
            guide_store_features(features + size_t(i) * kGuideIn, f);
            samples[i] = GuideSample{{r.wi[0], r.wi[1], r.wi[2]}, r.pb, r.w, {r.n[0], r.n[1], r.n[2]}};
            w = r.w;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        if ((threadIdx.x & 31) == 0 && w != 0.f) atomicAdd(wsum, w);
    }
}

__global__ void k_guide_norm(const int *rows, const float *wsum, float *wnorm, float *scale, int *stepDev) {
    const int n = *rows;
    const float s = *wsum;
    *wnorm = (n > 0 && s > 0.f) ? float(n) / s : 0.f;
    *scale = n > 0 ? 1.f / float(n) : 0.f;
    if (n > 0) ++*stepDev;  // this batch's Adam step
}

int guide_status(DeviceState &ds, GuideState &g) {
    int s = 0;
    PRB_CUDA(cudaMemcpyAsync(&s, g.status.ptr, sizeof(int), cudaMemcpyDeviceToHost, ds.stream));
    PRB_CUDA(cudaStreamSynchronize(ds.stream));
    return s;
}

// Fresh weights: He-uniform, the constant units' outgoing columns (biases) and the rows that
// produce a constant unit (or an unused output) zero.
std::vector<float> guide_init_weights(uint64_t seed) {
    std::vector<float> w(kGuideParams, 0.f);
    uint64_t st = seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    auto uni = [&]() {
        st ^= st >> 12;
        st ^= st << 25;
        st ^= st >> 27;
        return double((st * 0x2545F4914F6CDD1Dull) >> 11) * (1.0 / 9007199254740992.0);
    };
    for (int l = 0; l < kGuideLayers; ++l) {
        const int K = guide_layer_in(l), N = guide_layer_out(l);
        const double lim = std::sqrt(6.0 / double(l == 0 ? kGuideConstIn + 1 : K));
        for (int o = 0; o < N; ++o)
            for (int k = 0; k < K; ++k) {
                bool zero = (l == 0 && k >= kGuideConstIn) || (l > 0 && k == kGuideConstHid) ||
                            (l < kGuideLayers - 1 && o == kGuideConstHid) || (l == kGuideLayers - 1 && o > 40);
                w[size_t(guide_weight_offset(l)) + size_t(o) * K + k] = zero ? 0.f : float((2.0 * uni() - 1.0) * lim);
            }
    }
    return w;
}

void guide_prepare(DeviceState &ds, int device, bool reset, uint64_t seed) {
    GuideState &g = gGuide[device];
    const bool fresh = !g.ready;
    guide_setup(ds, g);
    if (fresh || reset) {
        std::vector<float> w = guide_init_weights(seed);
        guide_set_weights(ds, g, w.data());
        PRB_CUDA(cudaStreamSynchronize(ds.stream));
    }
}

bool guide_failed(DeviceState &ds, int device) {
    GuideState &g = gGuide[device];
    if (!g.ready) return false;
    int s = guide_status(ds, g);
    if (s) PRB_CUDA(cudaMemsetAsync(g.status.ptr, 0, sizeof(int), ds.stream));
    return s != 0;
}

GuideOpts guide_options(int device) { return gGuide[device].opts; }
float guide_learning_rate(int device) { return gGuide[device].lr; }

size_t guide_training_bytes(int maxRows) {
    const size_t fb = size_t(maxRows) * kGuideIn * sizeof(__half), sb = size_t(maxRows) * sizeof(GuideSample);
    return ((fb + 255) & ~size_t(255)) + ((sb + 255) & ~size_t(255)) + 256;
}
void guide_reserve_training(int device, int maxRows) { gGuide[device].train.ensure(guide_training_bytes(maxRows)); }
const void *guide_training_buffer(int device) { return gGuide[device].train.ptr; }

void guide_infer_rows(cudaStream_t st, int device, const __half *features, const int *dcount, int maxRows, float *out) {
    guide_forward(st, gGuide[device], features, dcount, maxRows, out);
}

void guide_train_records(cudaStream_t st, int device, const GuideTrainRec *recs, const int *dcount, int offset,
                         int maxRows, float lr) {
    GuideState &g = gGuide[device];
    if (lr <= 0.f) lr = g.lr;
    const size_t fb = size_t(maxRows) * kGuideIn * sizeof(__half), sb = size_t(maxRows) * sizeof(GuideSample);
    g.train.ensure(guide_training_bytes(maxRows));
    auto *feat = g.train.as<__half>();
    auto *smp = reinterpret_cast<GuideSample *>(g.train.as<unsigned char>() + ((fb + 255) & ~size_t(255)));
    auto *stats = reinterpret_cast<float *>(g.train.as<unsigned char>() + ((fb + 255) & ~size_t(255)) +
                                            ((sb + 255) & ~size_t(255)));
    int *rows = reinterpret_cast<int *>(stats);
    float *wsum = stats + 1, *wnorm = stats + 2, *scale = stats + 3;
    PRB_CUDA(cudaMemsetAsync(stats, 0, 16, st));
    k_guide_prep<<<g.sms * 4, 128, 0, st>>>(recs, dcount, offset, maxRows, feat, smp, rows, wsum, g.opts.bands);
    k_guide_norm<<<1, 1, 0, st>>>(rows, wsum, wnorm, scale, g.stepDev.as<int>());
    const int tiles = (maxRows + kTileRows - 1) / kTileRows;
    PRB_CUDA(cudaMemsetAsync(g.grad.ptr, 0, kGuideParams * sizeof(float), st));
    PRB_CUDA(cudaMemsetAsync(g.loss.ptr, 0, sizeof(float), st));
    k_guide_train<<<std::max(1, std::min(tiles, g.sms)), 128, train_smem(), st>>>(
        feat, smp, rows, g.packed.as<__half>(), g.grad.as<float>(), g.loss.as<float>(), g.status.as<int>(), wnorm,
        g.opts);
    k_guide_adam<<<64, 256, 0, st>>>(g.master.as<float>(), g.m.as<float>(), g.v.as<float>(), g.grad.as<float>(), 0.f,
                                     scale, lr, 0.9f, 0.999f, 1e-8f, g.stepDev.as<int>());
    k_guide_pack<<<64, 256, 0, st>>>(g.master.as<float>(), g.packed.as<__half>());
    count_launch(5);
}

} // namespace prb

using namespace prb;

namespace {

// Copies FP32 feature rows [n x 128] in as FP16 (scratch), with the row count on the device.
void stage_features(DeviceState &ds, GuideState &g, int64_t n, const float *features, size_t extraBytes,
                    __half **fh, int **dcount, unsigned char **extra) {
    size_t fb = size_t(n) * kGuideIn * sizeof(__half), f32 = size_t(n) * kGuideIn * sizeof(float);
    size_t need = ((fb + 255) & ~size_t(255)) + ((f32 + 255) & ~size_t(255)) + 256 + ((extraBytes + 255) & ~size_t(255));
    g.scratch.ensure(need);
    unsigned char *p = g.scratch.as<unsigned char>();
    *fh = reinterpret_cast<__half *>(p);
    float *f32buf = reinterpret_cast<float *>(p + ((fb + 255) & ~size_t(255)));
    *dcount = reinterpret_cast<int *>(p + ((fb + 255) & ~size_t(255)) + ((f32 + 255) & ~size_t(255)));
    *extra = p + ((fb + 255) & ~size_t(255)) + ((f32 + 255) & ~size_t(255)) + 256;
    PRB_CUDA(cudaMemcpyAsync(f32buf, features, f32, cudaMemcpyHostToDevice, ds.stream));
    int ni = int(n);
    PRB_CUDA(cudaMemcpyAsync(*dcount, &ni, sizeof(int), cudaMemcpyHostToDevice, ds.stream));
    k_guide_to_half<<<256, 256, 0, ds.stream>>>(f32buf, *fh, int(n * kGuideIn));
    count_launch();
    PRB_CUDA(cudaStreamSynchronize(ds.stream));
}

template <typename F> int guarded(char *err, int errLen, F &&f) {
    std::lock_guard<std::mutex> lock(gApiMutex);
    try {
        return f();
    } catch (const CudaError &ex) {
        set_err(err, errLen, ex.msg);
        return 1;
    } catch (const std::exception &ex) {
        set_err(err, errLen, ex.what());
        return 1;
    }
}

} // namespace

PRGPU_API int prgpu_guide_set_weights(int deviceIndex, const float *weights, char *err, int errLen) {
    return guarded(err, errLen, [&]() {
        if (!weights || deviceIndex < 0 || deviceIndex >= 64) {
            set_err(err, errLen, "bad arguments");
            return 1;
        }
        DeviceState &ds = device_state(deviceIndex);
        GuideState &g = gGuide[deviceIndex];
        guide_setup(ds, g);
        guide_set_weights(ds, g, weights);
        PRB_CUDA(cudaStreamSynchronize(ds.stream));
        return 0;
    });
}

PRGPU_API int prgpu_guide_get_weights(int deviceIndex, float *weights, char *err, int errLen) {
    return guarded(err, errLen, [&]() {
        if (!weights || deviceIndex < 0 || deviceIndex >= 64 || !gGuide[deviceIndex].ready) {
            set_err(err, errLen, "no guide weights on this device");
            return 1;
        }
        DeviceState &ds = device_state(deviceIndex);
        PRB_CUDA(cudaMemcpyAsync(weights, gGuide[deviceIndex].master.ptr, kGuideParams * sizeof(float),
                                 cudaMemcpyDeviceToHost, ds.stream));
        PRB_CUDA(cudaStreamSynchronize(ds.stream));
        return 0;
    });
}

PRGPU_API int prgpu_guide_infer(int deviceIndex, int64_t n, const float *features, float *out, char *err, int errLen) {
    return guarded(err, errLen, [&]() {
        if (deviceIndex < 0 || deviceIndex >= 64 || !gGuide[deviceIndex].ready) {
            set_err(err, errLen, "no guide weights on this device");
            return 1;
        }
        if (n < 0 || n > (int64_t(1) << 24) || (n > 0 && (!features || !out))) {
            set_err(err, errLen, "bad row count or null buffer");
            return 1;
        }
        if (n == 0) return 0;
        DeviceState &ds = device_state(deviceIndex);
        GuideState &g = gGuide[deviceIndex];
        __half *fh;
        int *dc;
        unsigned char *extra;
        stage_features(ds, g, n, features, size_t(n) * kGuideOut * sizeof(float), &fh, &dc, &extra);
        float *dout = reinterpret_cast<float *>(extra);
        PRB_CUDA(cudaMemsetAsync(g.status.ptr, 0, sizeof(int), ds.stream));
        guide_forward(ds.stream, g, fh, dc, int(n), dout);
        PRB_CUDA(cudaMemcpyAsync(out, dout, size_t(n) * kGuideOut * sizeof(float), cudaMemcpyDeviceToHost, ds.stream));
        PRB_CUDA(cudaStreamSynchronize(ds.stream));
        PRB_CUDA(cudaGetLastError());
        if (guide_status(ds, g)) {
            set_err(err, errLen, "guide kernel timed out waiting for the tensor cores");
            return 1;
        }
        return 0;
    });
}

PRGPU_API int prgpu_guide_gradient(int deviceIndex, int64_t n, const float *features, const float *samples,
                                   float *lossSum, float *grad, char *err, int errLen) {
    return guarded(err, errLen, [&]() {
        if (deviceIndex < 0 || deviceIndex >= 64 || !gGuide[deviceIndex].ready) {
            set_err(err, errLen, "no guide weights on this device");
            return 1;
        }
        if (n <= 0 || n > (int64_t(1) << 24) || !features || !samples || !grad) {
            set_err(err, errLen, "bad row count or null buffer");
            return 1;
        }
        DeviceState &ds = device_state(deviceIndex);
        GuideState &g = gGuide[deviceIndex];
        __half *fh;
        int *dc;
        unsigned char *extra;
        stage_features(ds, g, n, features, size_t(n) * sizeof(GuideSample), &fh, &dc, &extra);
        auto *ds_ = reinterpret_cast<GuideSample *>(extra);
        PRB_CUDA(cudaMemcpyAsync(ds_, samples, size_t(n) * sizeof(GuideSample), cudaMemcpyHostToDevice, ds.stream));
        PRB_CUDA(cudaMemsetAsync(g.status.ptr, 0, sizeof(int), ds.stream));
        guide_train(ds.stream, g, fh, ds_, dc, int(n));
        PRB_CUDA(cudaMemcpyAsync(grad, g.grad.ptr, kGuideParams * sizeof(float), cudaMemcpyDeviceToHost, ds.stream));
        float l = 0.f;
        PRB_CUDA(cudaMemcpyAsync(&l, g.loss.ptr, sizeof(float), cudaMemcpyDeviceToHost, ds.stream));
        PRB_CUDA(cudaStreamSynchronize(ds.stream));
        PRB_CUDA(cudaGetLastError());
        if (lossSum) *lossSum = l;
        if (guide_status(ds, g)) {
            set_err(err, errLen, "guide kernel timed out waiting for the tensor cores");
            return 1;
        }
        return 0;
    });
}

PRGPU_API int prgpu_guide_set_learning_rate(int deviceIndex, float learningRate, char *err, int errLen) {
    return guarded(err, errLen, [&]() {
        if (deviceIndex < 0 || deviceIndex >= 64 || !(learningRate > 0.f) || learningRate > 1.f) {
            set_err(err, errLen, "bad device or learning rate");
            return 1;
        }
        gGuide[deviceIndex].lr = learningRate;
        return 0;
    });
}

PRGPU_API int prgpu_guide_set_options(int deviceIndex, const prgpu::GuideOptions *opts, char *err, int errLen) {
    return guarded(err, errLen, [&]() {
        if (deviceIndex < 0 || deviceIndex >= 64) {
            set_err(err, errLen, "bad device");
            return 1;
        }
        GuideOpts o;  // null: the defaults
        if (opts) {
            if (!(opts->maxSelect > 0.f && opts->maxSelect <= 0.99f) || !(opts->logKappaMax >= 0.f && opts->logKappaMax <= 8.f) ||
                (opts->selectLoss != 0 && opts->selectLoss != 1) || opts->trainPasses < 1 || opts->trainPasses > 64 ||
                opts->bands < 0 || opts->bands > kGuideBandsMax || !(opts->weightClamp >= 0.f)) {
                set_err(err, errLen, "guide options out of range (0 < maxSelect <= 0.99, 0 <= logKappaMax <= 8, "
                                     "selectLoss 0 or 1, 1 <= trainPasses <= 64, 0 <= bands <= 12, weightClamp >= 0)");
                return 1;
            }
            o.maxSelect = opts->maxSelect;
            o.logKappaMax = opts->logKappaMax;
            o.selectLoss = opts->selectLoss;
            o.trainPasses = opts->trainPasses;
            o.bands = opts->bands;
            o.weightClamp = opts->weightClamp;
        }
        gGuide[deviceIndex].opts = o;
        return 0;
    });
}

PRGPU_API int prgpu_guide_get_options(int deviceIndex, prgpu::GuideOptions *out, char *err, int errLen) {
    return guarded(err, errLen, [&]() {
        if (deviceIndex < 0 || deviceIndex >= 64 || !out) {
            set_err(err, errLen, "bad arguments");
            return 1;
        }
        const GuideOpts &o = gGuide[deviceIndex].opts;
        out->maxSelect = o.maxSelect;
        out->logKappaMax = o.logKappaMax;
        out->selectLoss = o.selectLoss;
        out->trainPasses = o.trainPasses;
        out->bands = o.bands;
        out->weightClamp = o.weightClamp;
        return 0;
    });
}

PRGPU_API int prgpu_guide_stats(int deviceIndex, float *out4, char *err, int errLen) {
    return guarded(err, errLen, [&]() {
        if (!out4 || deviceIndex < 0 || deviceIndex >= 64 || !gGuide[deviceIndex].ready) {
            set_err(err, errLen, "no guide weights on this device");
            return 1;
        }
        DeviceState &ds = device_state(deviceIndex);
        GuideState &g = gGuide[deviceIndex];
        float loss = 0.f, tr[4] = {0.f, 0.f, 0.f, 0.f};
        int steps = 0;
        PRB_CUDA(cudaMemcpyAsync(&loss, g.loss.ptr, sizeof(float), cudaMemcpyDeviceToHost, ds.stream));
        PRB_CUDA(cudaMemcpyAsync(&steps, g.stepDev.ptr, sizeof(int), cudaMemcpyDeviceToHost, ds.stream));
        if (g.train.ptr) {
            // rows (int bits), weight sum of the last online batch: the stats block after the samples
            const size_t fb = size_t(1 << 16) * kGuideIn * sizeof(__half), sb = size_t(1 << 16) * sizeof(GuideSample);
            if (g.train.bytes >= ((fb + 255) & ~size_t(255)) + ((sb + 255) & ~size_t(255)) + 16)
                PRB_CUDA(cudaMemcpyAsync(tr, g.train.as<unsigned char>() + ((fb + 255) & ~size_t(255)) +
                                                 ((sb + 255) & ~size_t(255)),
                                         sizeof(tr), cudaMemcpyDeviceToHost, ds.stream));
        }
        PRB_CUDA(cudaStreamSynchronize(ds.stream));
        int rows;
        std::memcpy(&rows, &tr[0], sizeof(int));
        out4[0] = loss;
        out4[1] = float(rows);
        out4[2] = tr[1];
        out4[3] = float(steps);
        return 0;
    });
}

PRGPU_API int prgpu_guide_adam_step(int deviceIndex, float gradScale, float learningRate, char *err, int errLen) {
    return guarded(err, errLen, [&]() {
        if (deviceIndex < 0 || deviceIndex >= 64 || !gGuide[deviceIndex].ready) {
            set_err(err, errLen, "no guide weights on this device");
            return 1;
        }
        DeviceState &ds = device_state(deviceIndex);
        guide_adam(ds.stream, gGuide[deviceIndex], gradScale, learningRate);
        PRB_CUDA(cudaStreamSynchronize(ds.stream));
        return 0;
    });
}
