// Verification entry points: the device BxDF, phase-function and homogeneous-medium code of the
// path tracer evaluated on caller-supplied inputs, with the input/output layouts of the oracle
// harness, so that identical inputs can be compared against the reference implementations
// (src/materials/bxdf.cpp:64-256, src/media/medium.cpp:15-103).

#include <vector>

#include "bsdf.cuh"
#include "layered.cuh"
#include "device.cuh"
#include "lights.cuh"

namespace prb {

// params (16): R[4] | eta[4] | k[4] | etaD, alphaX, alphaY, mode (0 radiance, 1 importance)
// in (9 per item): wo[3], wi[3], uc, u0, u1
// out (16 per item): f[4], pdf, sample ok, f[4], pdf, wi[3], flags, eta
__global__ void k_eval_bxdf(int kind, Lobe lobe, bool radiance, int64_t n, const float *__restrict__ in,
                            float *__restrict__ out) {
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < n; j += int64_t(gridDim.x) * blockDim.x) {
        const float *x = in + 9 * j;
        float *y = out + 16 * j;
        V3 wo = mk(x[0], x[1], x[2]), wi = mk(x[3], x[4], x[5]);
        SS f = lobe_f(lobe, wo, wi, radiance);
        for (int i = 0; i < 4; ++i) y[i] = f.v[i];
        y[4] = lobe_pdf(lobe, wo, wi);
        for (int i = 5; i < 16; ++i) y[i] = 0.f;
        BSample s;
        if (lobe_sample(lobe, wo, x[6], x[7], x[8], &s, radiance)) {
            y[5] = 1.f;
            for (int i = 0; i < 4; ++i) y[6 + i] = s.f.v[i];
            y[10] = s.pdf;
            y[11] = s.wi.x;
            y[12] = s.wi.y;
            y[13] = s.wi.z;
            y[14] = float(s.flags);
            y[15] = s.eta;
        }
    }
}

// The coated / sheen BSDF on local-frame inputs (same in / out layout as k_eval_bxdf; out[15] is
// 1 when the sampled pdf is only proportional).
__global__ void k_eval_full(FullBsdf b, int64_t n, const float *__restrict__ in, float *__restrict__ out) {
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < n; j += int64_t(gridDim.x) * blockDim.x) {
        const float *x = in + 9 * j;
        float *y = out + 16 * j;
        V3 wo = mk(x[0], x[1], x[2]), wi = mk(x[3], x[4], x[5]);
        SS f = full_f(b, wo, wi);
        for (int i = 0; i < 4; ++i) y[i] = f.v[i];
        y[4] = full_pdf(b, wo, wi);
        for (int i = 5; i < 16; ++i) y[i] = 0.f;
        BSample s;
        bool proportional = false;
        if (full_sample(b, wo, x[6], x[7], x[8], &s, &proportional)) {
            y[5] = 1.f;
            for (int i = 0; i < 4; ++i) y[6 + i] = s.f.v[i];
            y[10] = s.pdf;
            y[11] = s.wi.x;
            y[12] = s.wi.y;
            y[13] = s.wi.z;
            y[14] = float(s.flags);
            y[15] = proportional ? 1.f : 0.f;
        }
    }
}

// in (7 per item): cosTheta, g, wo[3], u0, u1; out (5 per item): p(cosTheta), wi[3], pdf
__global__ void k_eval_phase(int64_t n, const float *__restrict__ in, float *__restrict__ out) {
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < n; j += int64_t(gridDim.x) * blockDim.x) {
        const float *x = in + 7 * j;
        float *y = out + 5 * j;
        y[0] = hg_phase(x[0], x[1]);
        float pdf;
        V3 wi = hg_sample(mk(x[2], x[3], x[4]), x[1], x[5], x[6], &pdf);
        y[1] = wi.x;
        y[2] = wi.y;
        y[3] = wi.z;
        y[4] = pdf;
    }
}

// Homogeneous medium, sigma_a / sigma_s given at the 4 wavelengths.
// in (10 per item): sa[4], ss[4], tMax, u; out (14 per item): Tr(tMax)[4], scattered, t,
// weight[4], pdfRatio[4] -- the hero-driven free-flight sampling of the path tracer.
__global__ void k_eval_homogeneous(int64_t n, const float *__restrict__ in, float *__restrict__ out) {
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < n; j += int64_t(gridDim.x) * blockDim.x) {
        const float *x = in + 10 * j;
        float *y = out + 14 * j;
        SS sa{{x[0], x[1], x[2], x[3]}}, ss{{x[4], x[5], x[6], x[7]}};
        SS st = sa + ss;
        float tMax = x[8];
        SS Tm;
        for (int i = 0; i < 4; ++i) Tm.v[i] = isinf(tMax) ? (st.v[i] > 0.f ? 0.f : 1.f) : expf(-st.v[i] * tMax);
        for (int i = 0; i < 4; ++i) y[i] = Tm.v[i];
        float u = fminf(x[9], kOneMinusEps);
        float t = st.v[0] > 0.f ? -logf(1.f - u) / st.v[0] : kInf;
        SS w = splat(0.f), r = splat(1.f);
        if (t < tMax) {
            SS T;
            for (int i = 0; i < 4; ++i) T.v[i] = expf(-st.v[i] * t);
            float pdf0 = st.v[0] * T.v[0];
            y[4] = 1.f;
            y[5] = t;
            if (pdf0 > 0.f) {
                w = T * ss * (1.f / pdf0);
                r = st * T * (1.f / pdf0);
            }
        } else {
            y[4] = 0.f;
            y[5] = tMax;
            if (Tm.v[0] > 0.f) {
                w = Tm * (1.f / Tm.v[0]);
                r = w;
            }
        }
        for (int i = 0; i < 4; ++i) {
            y[6 + i] = w.v[i];
            y[10 + i] = r.v[i];
        }
    }
}

// Light-BVH selection at shading points: in 7 floats (p[3], n[3], u), out 2 floats (light, pmf),
// and optionally the pmf of every light at that point.
__global__ void k_eval_light_bvh(LightTree t, int lightCount, int64_t n, const float *__restrict__ in,
                                 float *__restrict__ out, float *__restrict__ pmfOut) {
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < n; j += int64_t(gridDim.x) * blockDim.x) {
        const float *x = in + 7 * j;
        V3 p = mk(x[0], x[1], x[2]), nn = mk(x[3], x[4], x[5]);
        float pmf = 0.f;
        int li = lbvh_sample(t, p, nn, x[6], &pmf);
        out[2 * j] = float(li);
        out[2 * j + 1] = li >= 0 ? pmf : 0.f;
        if (pmfOut)
            for (int k = 0; k < lightCount; ++k) pmfOut[j * lightCount + k] = lbvh_pmf(t, k, p, nn);
    }
}

namespace {

template <typename Launch>
int run_eval(int deviceIndex, int64_t n, int inStride, int outStride, const float *in, float *out, char *err,
             int errLen, Launch launch) {
    std::lock_guard<std::mutex> lock(gApiMutex);
    if (n < 0 || (n > 0 && (!in || !out)) || n > (int64_t(1) << 26)) {
        set_err(err, errLen, "bad arguments");
        return 1;
    }
    if (n == 0) return 0;
    try {
        DeviceState &ds = device_state(deviceIndex);
        DevBuf din, dout;
        din.ensure(size_t(n) * inStride * sizeof(float));
        dout.ensure(size_t(n) * outStride * sizeof(float));
        PRB_CUDA(cudaMemcpyAsync(din.ptr, in, size_t(n) * inStride * sizeof(float), cudaMemcpyHostToDevice, ds.stream));
        int grid = int(std::min<int64_t>((n + 255) / 256, int64_t(ds.prop.multiProcessorCount) * 8));
        launch(grid, ds.stream, din.as<float>(), dout.as<float>());
        count_launch();
        PRB_CUDA(cudaGetLastError());
        PRB_CUDA(cudaMemcpyAsync(out, dout.ptr, size_t(n) * outStride * sizeof(float), cudaMemcpyDeviceToHost, ds.stream));
        PRB_CUDA(cudaStreamSynchronize(ds.stream));
        din.release();
        dout.release();
        return 0;
    } catch (const CudaError &e) {
        set_err(err, errLen, e.msg);
        return 1;
    }
}

} // namespace
} // namespace prb

using namespace prb;

PRGPU_API int prgpu_eval_bxdf(int deviceIndex, int kind, const float *params, int64_t n, const float *in, float *out,
                              char *err, int errLen) {
    if (!params || kind < 0 || kind > 3) {
        set_err(err, errLen, "bad BxDF kind or parameters");
        return 1;
    }
    Lobe l;
    l.kind = kind == 0 ? kLobeDiffuse : kind == 1 ? kLobeConductor : kind == 2 ? kLobeDielectric : kLobeThin;
    for (int i = 0; i < 4; ++i) {
        l.R.v[i] = params[i];
        l.eta.v[i] = params[4 + i];
        l.k.v[i] = params[8 + i];
    }
    l.etaD = params[12];
    // Alpha clamping of a rough distribution, as the material code does on construction.
    l.mf = Ggx{params[13], params[14]};
    if (!(std::max(l.mf.ax, l.mf.ay) < 1e-3f)) {
        l.mf.ax = std::max(l.mf.ax, 1e-4f);
        l.mf.ay = std::max(l.mf.ay, 1e-4f);
    }
    bool radiance = params[15] == 0.f;
    return run_eval(deviceIndex, n, 9, 16, in, out, err, errLen, [&](int g, cudaStream_t s, const float *i, float *o) {
        k_eval_bxdf<<<g, 256, 0, s>>>(kind, l, radiance, n, i, o);
    });
}

PRGPU_API int prgpu_eval_full_bsdf(int deviceIndex, const float *params, const float *sheenTable, int64_t n,
                                   const float *in, float *out, char *err, int errLen) {
    if (!params || params[1] < 0.f || params[1] > 2.f || (params[0] != 0.f && params[1] > 1.f) ||
        params[25] < 0.f || params[25] > 4096.f || params[26] < 0.f || params[26] > 4096.f ||
        (params[27] > 0.f && !sheenTable)) {
        set_err(err, errLen, "bad coated / sheen BSDF parameters");
        return 1;
    }
    auto ss = [&](int o) {
        SS v;
        for (int i = 0; i < 4; ++i) v.v[i] = params[o + i];
        return v;
    };
    auto ggx = [](float ax, float ay) {
        Ggx g{ax, ay};
        if (!(std::max(ax, ay) < 1e-3f)) {
            g.ax = std::max(ax, 1e-4f);
            g.ay = std::max(ay, 1e-4f);
        }
        return g;
    };
    const int kind = int(params[1]);
    Lobe base;
    base.kind = kind == 0 ? kLobeDiffuse : kind == 1 ? kLobeConductor : kLobeDielectric;
    base.R = ss(2);
    base.eta = ss(6);
    base.k = ss(10);
    base.etaD = params[14];
    base.mf = ggx(params[15], params[16]);
    FullBsdf b;
    b.black = false;
    b.layered = params[0] != 0.f;
    b.sheen = params[27] > 0.f;
    b.base = base;
    if (b.layered) {
        b.lay.top.kind = kLobeDielectric;
        b.lay.top.etaD = params[17];
        b.lay.top.mf = ggx(params[18], params[18]);
        b.lay.bottom = base;
        b.lay.thickness = std::max(params[19], 1.17549435e-38f);
        b.lay.g = params[20];
        b.lay.albedo = ss(21);
        b.lay.hasAlbedo = false;
        for (int i = 0; i < 4; ++i) b.lay.hasAlbedo = b.lay.hasAlbedo || b.lay.albedo.v[i] != 0.f;
        b.lay.maxDepth = int(params[25]);
        b.lay.nSamples = std::max(1, int(params[26]));
    }
    float *table = nullptr;
    if (b.sheen) {
        for (int i = 0; i < 4; ++i) b.sh.color.v[i] = std::max(0.f, params[29 + i]);
        b.sh.alpha = std::min(1.f, std::max(0.05f, params[28]));
        b.sh.weight = std::min(1.f, std::max(0.f, params[27]));
        float cmax = std::max(std::max(b.sh.color.v[0], b.sh.color.v[1]), std::max(b.sh.color.v[2], b.sh.color.v[3]));
        b.sh.colorMax = std::min(1.f, std::max(0.f, cmax));
        if (cudaMalloc(&table, sizeof(float) * kSheenAlphaBins * kSheenMuBins) != cudaSuccess ||
            cudaMemcpy(table, sheenTable, sizeof(float) * kSheenAlphaBins * kSheenMuBins, cudaMemcpyHostToDevice) !=
                cudaSuccess) {
            if (table) cudaFree(table);
            set_err(err, errLen, "sheen table upload failed");
            return 1;
        }
        b.sh.table = table;
    }
    int rc = run_eval(deviceIndex, n, 9, 16, in, out, err, errLen, [&](int g, cudaStream_t s, const float *i, float *o) {
        k_eval_full<<<g, 256, 0, s>>>(b, n, i, o);
    });
    if (table) cudaFree(table);
    return rc;
}

PRGPU_API int prgpu_eval_phase(int deviceIndex, int64_t n, const float *in, float *out, char *err, int errLen) {
    return run_eval(deviceIndex, n, 7, 5, in, out, err, errLen, [&](int g, cudaStream_t s, const float *i, float *o) {
        k_eval_phase<<<g, 256, 0, s>>>(n, i, o);
    });
}

PRGPU_API int prgpu_eval_homogeneous(int deviceIndex, int64_t n, const float *in, float *out, char *err, int errLen) {
    return run_eval(deviceIndex, n, 10, 14, in, out, err, errLen, [&](int g, cudaStream_t s, const float *i, float *o) {
        k_eval_homogeneous<<<g, 256, 0, s>>>(n, i, o);
    });
}

PRGPU_API int prgpu_eval_light_bvh(int deviceIndex, const prgpu::LightBVHNode *nodes, int32_t nodeCount,
                                   int32_t lightCount, float bvhProb, int64_t n, const float *in, float *out,
                                   float *pmfOut, char *err, int errLen) {
    std::lock_guard<std::mutex> lock(gApiMutex);
    if (!nodes || nodeCount <= 0 || lightCount <= 0 || n < 0 || (n > 0 && (!in || !out)) || n > (int64_t(1) << 22)) {
        set_err(err, errLen, "bad arguments");
        return 1;
    }
    std::vector<int> leafOf(size_t(lightCount), -1);
    for (int32_t i = 0; i < nodeCount; ++i) {
        const prgpu::LightBVHNode &b = nodes[i];
        if (b.light >= 0) {
            if (b.light >= lightCount) {
                set_err(err, errLen, "light BVH leaf out of range");
                return 1;
            }
            leafOf[size_t(b.light)] = i;
        } else if (b.child1 <= i + 1 || b.child1 >= nodeCount) {
            set_err(err, errLen, "malformed light BVH interior node");
            return 1;
        }
        if (b.parent >= i || b.parent < -1 || (i > 0 && b.parent < 0)) {
            set_err(err, errLen, "malformed light BVH parent link");
            return 1;
        }
    }
    if (n == 0) return 0;
    try {
        DeviceState &ds = device_state(deviceIndex);
        DevBuf dn, dl, din, dout, dpmf;
        dn.ensure(size_t(nodeCount) * sizeof(prgpu::LightBVHNode));
        dl.ensure(leafOf.size() * sizeof(int));
        din.ensure(size_t(n) * 7 * sizeof(float));
        dout.ensure(size_t(n) * 2 * sizeof(float));
        if (pmfOut) dpmf.ensure(size_t(n) * lightCount * sizeof(float));
        PRB_CUDA(cudaMemcpyAsync(dn.ptr, nodes, size_t(nodeCount) * sizeof(prgpu::LightBVHNode), cudaMemcpyHostToDevice, ds.stream));
        PRB_CUDA(cudaMemcpyAsync(dl.ptr, leafOf.data(), leafOf.size() * sizeof(int), cudaMemcpyHostToDevice, ds.stream));
        PRB_CUDA(cudaMemcpyAsync(din.ptr, in, size_t(n) * 7 * sizeof(float), cudaMemcpyHostToDevice, ds.stream));
        LightTree t{dn.as<prgpu::LightBVHNode>(), nodeCount, bvhProb, dl.as<int>()};
        int grid = int(std::min<int64_t>((n + 255) / 256, int64_t(ds.prop.multiProcessorCount) * 8));
        k_eval_light_bvh<<<grid, 256, 0, ds.stream>>>(t, lightCount, n, din.as<float>(), dout.as<float>(),
                                                       pmfOut ? dpmf.as<float>() : nullptr);
        count_launch();
        PRB_CUDA(cudaGetLastError());
        PRB_CUDA(cudaMemcpyAsync(out, dout.ptr, size_t(n) * 2 * sizeof(float), cudaMemcpyDeviceToHost, ds.stream));
        if (pmfOut)
            PRB_CUDA(cudaMemcpyAsync(pmfOut, dpmf.ptr, size_t(n) * lightCount * sizeof(float), cudaMemcpyDeviceToHost, ds.stream));
        PRB_CUDA(cudaStreamSynchronize(ds.stream));
        dn.release();
        dl.release();
        din.release();
        dout.release();
        dpmf.release();
        return 0;
    } catch (const CudaError &e) {
        set_err(err, errLen, e.msg);
        return 1;
    }
}
