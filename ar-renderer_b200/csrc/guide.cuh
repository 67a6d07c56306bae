// Path-guiding network: the parts shared by the tensor-core kernels (guide.cu) and the shading
// kernel -- input encoding, decoding of the network output into a von Mises-Fisher mixture plus
// a selection probability, the mixture's sampling and pdf, and the gradient of the training loss.
// No counterpart in the reference renderer (its PathIntegrator samples the BSDF only,
// src/integrators/path.cpp:215-224, the site where this guide is combined with it).
//
// Network: 128 inputs -> 4 hidden layers of 64 (ReLU) -> 48 outputs, FP16 weights and
// activations, FP32 accumulation. Biases are folded into the weights: input 81 and hidden unit 63
// of every hidden layer are held at 1, so the weight column of that unit is the next layer's bias.
//   inputs: x in [0,1]^3 (position normalised to the scene bounds), sin / cos(2^b pi x) for 12
//           bands b (72), shading normal (3), outgoing direction (3), 1, zeros to 128.
//   outputs: per lobe k < 8: direction (3, normalised), log kappa (clamped to [-4, 8]), weight
//           logit (softmax over the 8); output 40: selection logit, c = maxSelect sigmoid (default 0.5);
//           41..47 unused.
// One-sample MIS with the BSDF: wi ~ c q_n + (1 - c) p_bsdf, the pdf of both computed in FP32 from
// the same decoded parameters, so the estimator stays unbiased for any weights. q_n is the mixture
// folded onto the hemisphere of the shading normal n that holds wo (a sample below is mirrored
// across the tangent plane): q_n(w) = q(w) + q(w - 2 (w.n) n) there, 0 on the other side, so no
// guided sample is wasted below a reflecting surface.
// Loss per training sample (x, n, wo, wi, p_bsdf(wi), weight w >= 0), w = f cos Li / pdf_used:
//   -w log q_n(wi)                               (the lobes: KL divergence from the product of
//                                                 BSDF and incident light)
//   -w log(c q_n(wi) + (1 - c) p_bsdf(wi))       (the selection probability only: q_n held fixed)
// Training c through the mixture alone would let it collapse to 0 while the lobes are still poor,
// after which the lobes' gradient (proportional to c) vanishes.
#pragma once

#include <cuda_fp16.h>

#include <cstring>

#include "common.cuh"

namespace prb {

constexpr int kGuideIn = 128, kGuideHid = 64, kGuideOut = 48, kGuideLayers = 5, kGuideLobes = 8;
constexpr int kGuideBands = 12, kGuideBandsMax = 12, kGuideConstIn = 81, kGuideConstHid = 63;
// Weight matrix l is [out_l x in_l]; the flattened FP32 master array keeps them in order, row-major.
__host__ __device__ constexpr int guide_layer_in(int l) { return l == 0 ? kGuideIn : kGuideHid; }
__host__ __device__ constexpr int guide_layer_out(int l) { return l == kGuideLayers - 1 ? kGuideOut : kGuideHid; }
constexpr int kGuideParams = kGuideHid * kGuideIn + 3 * kGuideHid * kGuideHid + kGuideOut * kGuideHid;  // 23,552
constexpr int kGuideVertices = 4;  // diffuse vertices per path that are guided and recorded

// Settings of sampling and training (prgpu_guide_set_options). Defaults: c = 0.5 sigmoid, log kappa
// clamped to [-4, 8], c trained on the KL objective, the online batch's weights (normalised to mean
// 1) clamped at 20 -- the best of the settings measured on the slit and indirectly lit box scenes.
struct GuideOpts {
    float maxSelect = 0.5f;    // c = maxSelect * sigmoid(output 40)
    float logKappaMax = 8.f;   // upper clamp of log kappa
    int selectLoss = 0;        // c's objective: 0 = -w log p_mix, 1 = second moment w^2 / p_mix
    int trainPasses = 1;       // passes over each chunk's recorded samples (online training)
    int bands = kGuideBandsMax;  // position encoding bands in use (the rest of the inputs zero)
    float weightClamp = 20.f;  // > 0: online training weights (normalised to mean 1 per batch) clamped to it
};

__host__ __device__ constexpr int guide_weight_offset(int l) {
    return l == 0 ? 0 : kGuideHid * kGuideIn + (l - 1) * kGuideHid * kGuideHid;
}

// Input features (FP32) of a shading point; bmin / bext: scene bounds and extent; bands: the
// encoding bands in use (higher bands' inputs are zero).
__device__ __forceinline__ void guide_features(V3 x, V3 n, V3 wo, const float *bmin, const float *bext, float *f,
                                               int bands = kGuideBands) {
    float xn[3] = {(x.x - bmin[0]) / bext[0], (x.y - bmin[1]) / bext[1], (x.z - bmin[2]) / bext[2]};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        xn[a] = fminf(fmaxf(xn[a], 0.f), 1.f);
        f[a] = xn[a];
    }
#pragma unroll
    for (int b = 0; b < kGuideBands; ++b)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float s, c;
            sincospif(xn[a] * float(1 << b), &s, &c);
            f[3 + 6 * b + 2 * a] = b < bands ? s : 0.f;
            f[3 + 6 * b + 2 * a + 1] = b < bands ? c : 0.f;
        }
    f[75] = n.x, f[76] = n.y, f[77] = n.z;
    f[78] = wo.x, f[79] = wo.y, f[80] = wo.z;
    f[kGuideConstIn] = 1.f;
}

// One row of FP16 features as 16-byte stores (8 features each): rows are 256 bytes apart, so
// narrower stores would each fill only a few bytes of a memory sector.
__device__ __forceinline__ void guide_store_features(__half *row, const float *f) {
    int4 *dst = reinterpret_cast<int4 *>(row);
#pragma unroll
    for (int k = 0; k < kGuideIn / 8; ++k) {
        __half2 h[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) h[e] = __floats2half2_rn(f[8 * k + 2 * e], f[8 * k + 2 * e + 1]);
        int4 v;
        memcpy(&v, h, sizeof(v));
        dst[k] = v;
    }
}

struct GuideMix {
    V3 mu[kGuideLobes];
    float kappa[kGuideLobes];
    float pi[kGuideLobes];
    float c;
};

__device__ __forceinline__ float guide_sigmoid(float x) { return 1.f / (1.f + expf(-x)); }

__device__ __forceinline__ GuideMix guide_decode(const float *o, const GuideOpts &op) {
    GuideMix m;
    float mx = -1e30f;
#pragma unroll
    for (int k = 0; k < kGuideLobes; ++k) mx = fmaxf(mx, o[5 * k + 4]);
    float sum = 0.f;
#pragma unroll
    for (int k = 0; k < kGuideLobes; ++k) {
        V3 v = mk(o[5 * k], o[5 * k + 1], o[5 * k + 2]);
        float l = sqrtf(dot(v, v));
        m.mu[k] = l > 1e-6f ? v * (1.f / l) : mk(0.f, 0.f, 1.f);
        m.kappa[k] = expf(fminf(fmaxf(o[5 * k + 3], -4.f), op.logKappaMax));
        m.pi[k] = expf(o[5 * k + 4] - mx);
        sum += m.pi[k];
    }
#pragma unroll
    for (int k = 0; k < kGuideLobes; ++k) m.pi[k] /= sum;
    m.c = op.maxSelect * guide_sigmoid(o[40]);
    return m;
}

// vMF density kappa / (2 pi (1 - exp(-2 kappa))) exp(kappa (mu.w - 1)) (normalised on the sphere).
__device__ __forceinline__ float vmf_pdf(V3 mu, float kappa, V3 w) {
    float t = dot(mu, w) - 1.f;
    if (kappa < 1e-4f) return kInv4Pi;
    return kappa / (2.f * kPi * -expm1f(-2.f * kappa)) * expf(kappa * t);
}

__device__ __forceinline__ float guide_pdf(const GuideMix &m, V3 w) {
    float q = 0.f;
#pragma unroll
    for (int k = 0; k < kGuideLobes; ++k) q += m.pi[k] * vmf_pdf(m.mu[k], m.kappa[k], w);
    return q;
}

__device__ __forceinline__ V3 guide_mirror(V3 w, V3 n) { return w - n * (2.f * dot(w, n)); }

// The folded mixture pdf q_n(w); side: +1 / -1 = the hemisphere of n that holds wo.
__device__ __forceinline__ float guide_pdf_folded(const GuideMix &m, V3 w, V3 n, float side) {
    if (dot(w, n) * side <= 0.f) return 0.f;
    return guide_pdf(m, w) + guide_pdf(m, guide_mirror(w, n));
}

// Lobe by u0 over the weights, then the vMF sample of W. Jakob, "Numerically stable sampling of
// the von Mises-Fisher distribution on S^2" (2012): cos theta = 1 + log(u + (1 - u) e^{-2 kappa}) / kappa.
__device__ __forceinline__ V3 guide_sample(const GuideMix &m, float u0, float u1, float u2) {
    int k = kGuideLobes - 1;
    float acc = 0.f;
#pragma unroll
    for (int i = 0; i < kGuideLobes; ++i) {
        acc += m.pi[i];
        if (u0 < acc) {
            k = i;
            break;
        }
    }
    float kap = m.kappa[k];
    float ct = kap < 1e-4f ? 1.f - 2.f * u1 : 1.f + logf(u1 + (1.f - u1) * expf(-2.f * kap)) / kap;
    ct = fminf(fmaxf(ct, -1.f), 1.f);
    float st = sqrtf(fmaxf(0.f, 1.f - ct * ct));
    float sp, cp;
    sincospif(2.f * u2, &sp, &cp);
    V3 t, b;
    V3 mu = m.mu[k];
    // Orthonormal basis around mu (Duff et al. 2017, "Building an orthonormal basis, revisited").
    float sgn = copysignf(1.f, mu.z);
    float a = -1.f / (sgn + mu.z), bb = mu.x * mu.y * a;
    t = mk(1.f + sgn * mu.x * mu.x * a, sgn * bb, -sgn * mu.x);
    b = mk(bb, sgn + mu.y * mu.y * a, -mu.y);
    return t * (st * cp) + b * (st * sp) + mu * ct;
}

// A training sample recorded by the renderer: normalised position, shading normal, outgoing and
// sampled directions, the BSDF pdf of wi and the weight w = f cos Li / pdf_used (luminance-free:
// the average over the hero wavelengths).
struct GuideTrainRec {
    float xn[3], n[3], wo[3], wi[3], pb, w;
};

// Input features from a normalised position (x already in [0,1]^3).
__device__ __forceinline__ void guide_features_n(const float *xn, V3 n, V3 wo, float *f, int bands = kGuideBands) {
    const float zero[3] = {0.f, 0.f, 0.f}, one[3] = {1.f, 1.f, 1.f};
    guide_features(mk(xn[0], xn[1], xn[2]), n, wo, zero, one, f, bands);
}

// Gradient of the two-part loss above with respect to the 48 raw outputs (FP32): lobe outputs
// from -w log q_n, the selection output from -w log(c q_n + (1 - c) pb) with q_n fixed. wi lies on
// the side of n the sample came from, so q_n(wi) = q(wi) + q(mirror(wi)). Returns the sum of both
// parts; g receives the gradient (zero for the unused outputs 41..47).
// With op.selectLoss = 1 the selection output instead descends the second moment of the one-sample
// estimator f Li / p_mix, E[(f Li)^2 / p_mix]: its derivative in c, estimated from a sample drawn
// from p_mix with w = f Li / p_mix, is -w^2 (q_n - pb) / p_mix (the variance-optimal selection
// rather than the KL-optimal one).
__device__ __forceinline__ float guide_loss_grad(const float *o, V3 wi, V3 n, float pb, float w, float *g,
                                                 const GuideOpts &op) {
#pragma unroll
    for (int i = 0; i < kGuideOut; ++i) g[i] = 0.f;
    GuideMix m = guide_decode(o, op);
    const V3 wr = guide_mirror(wi, n);
    float v1[kGuideLobes], v2[kGuideLobes];
    float q = 0.f;
#pragma unroll
    for (int k = 0; k < kGuideLobes; ++k) {
        v1[k] = vmf_pdf(m.mu[k], m.kappa[k], wi);
        v2[k] = vmf_pdf(m.mu[k], m.kappa[k], wr);
        q += m.pi[k] * (v1[k] + v2[k]);
    }
    float p = m.c * q + (1.f - m.c) * pb;
    if (!(p > 0.f) || !(q > 0.f) || !(w > 0.f)) return 0.f;
    // The selection term's weight: w (KL), or w^2 for the second moment (the surrogate
    // -w w' log p with w' = w held fixed, whose c-derivative is -w^2 (q_n - pb) / p).
    const float ws = op.selectLoss == 1 ? w * w : w;
    float loss = -w * logf(q) - ws * logf(p);
    float dq = -w / q;                             // d(-w log q_n)/dq_n
    float dc = -ws * (q - pb) / p;                 // d(-ws log p)/dc at fixed q_n
    float s = guide_sigmoid(o[40]);
    g[40] = dc * op.maxSelect * s * (1.f - s);
    float sumPiG = 0.f;
#pragma unroll
    for (int k = 0; k < kGuideLobes; ++k) sumPiG += m.pi[k] * dq * (v1[k] + v2[k]);
#pragma unroll
    for (int k = 0; k < kGuideLobes; ++k) {
        // softmax weights
        g[5 * k + 4] = m.pi[k] * dq * (v1[k] + v2[k]) - m.pi[k] * sumPiG;
        const float d1 = dq * m.pi[k] * v1[k], d2 = dq * m.pi[k] * v2[k];  // dL/d(log vmf_k) at wi, wr
        const float kap = m.kappa[k];
        const float raw = o[5 * k + 3];
        if (raw > -4.f && raw < op.logKappaMax && kap >= 1e-4f) {
            // d log vmf / d kappa = 1/kappa - 2 e^{-2k} / (1 - e^{-2k}) + (mu.w - 1); d kappa / d raw = kappa
            const float base = 1.f / kap - 2.f * expf(-2.f * kap) / (-expm1f(-2.f * kap));
            g[5 * k + 3] = (d1 * (base + dot(m.mu[k], wi) - 1.f) + d2 * (base + dot(m.mu[k], wr) - 1.f)) * kap;
        }
        // d log vmf / d mu = kappa w; mu = v / |v|: dmu/dv = (I - mu mu^T) / |v|
        V3 v = mk(o[5 * k], o[5 * k + 1], o[5 * k + 2]);
        float l = sqrtf(dot(v, v));
        if (l > 1e-6f) {
            V3 gm = (wi * d1 + wr * d2) * kap;
            V3 gv = (gm - m.mu[k] * dot(m.mu[k], gm)) * (1.f / l);
            g[5 * k] = gv.x, g[5 * k + 1] = gv.y, g[5 * k + 2] = gv.z;
        }
    }
    return loss;
}

} // namespace prb
