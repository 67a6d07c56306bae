// The wavefront path tracer's device side: path state in structure-of-arrays form, the per-bounce
// kernels and the film kernel, used by the single-render and the batched drivers of render.cu (the
// one file that includes it: the kernels have external linkage).
//
// The estimator is the reference's pr::PathIntegrator::Li (src/integrators/path.cpp:113-238) as its
// GPU module restates it (src/gpu/prender_gpu.cpp:1344-1460): 4 hero wavelengths, next-event
// estimation with power-heuristic MIS, path-level spectral MIS in homogeneous media (rPath, the
// hero-driven free-flight pdf ratios, with Lhero kept for paths whose secondary wavelengths a
// dispersive interface terminates), Russian roulette on the MIS-weighted throughput from the
// third vertex on, no clamping unless the caller asks for it.
//
// Instead of one thread looping over a pixel's whole path (the reference megakernel), a batch of
// paths lives in structure-of-arrays state in HBM and advances one bounce per round of kernels:
//   raygen  -> closest-hit (k_extend) -> shading (k_shade: media, emission, BSDF, NEE, RR)
//           -> shadow rays (k_shadow) -> ... until the queue is empty -> film (k_film).
// Queues are compacted with warp-aggregated atomics (one atomic per warp, slots handed out by
// ballot + popc), so every kernel reads a dense index list. Each path's final XYZ is added to an
// FP64 per-pixel film in sample-index order, one sample at a time: a render split into batches
// produces the same bits as one uninterrupted render.
//
// Batched form (kBatch): paths of many renders share the queues; each path carries its render's
// index in bits 24..31 of meta.w and reads that render's DevScene from a device table.
#pragma once

#include <cmath>

#include "bsdf.cuh"
#include "guide.cuh"
#include "layered.cuh"
#include "lights.cuh"
#include "media.cuh"
#include "noise.cuh"
#include "scene.cuh"

namespace prb {
// ---------------------------------------------------------------------------------------------
// Path state (structure of arrays, 16-byte vector accesses)

struct Paths {
    float4 *o;       // origin, w: prevPdf
    float4 *d;       // direction, w: etaScale
    float4 *beta;    // throughput per wavelength
    float4 *rpath;   // spectral MIS pdf ratios
    float4 *L;       // MIS-weighted radiance
    float4 *Lhero;   // unweighted radiance (valid once secondaries terminate)
    float4 *lam;     // wavelengths
    float4 *lpdf;    // wavelength pdfs
    ulonglong2 *rng; // PCG32 state, increment
    int4 *meta;      // pixel, depth, medium, flags (bit 0 specular, bits 8..23 interface crossings)
    float4 *prevP;   // previous scattering vertex, w: filter weight of the camera sample
    float4 *prevN;   // geometric normal there (0 in media), w: iteration guard (int bits)
    float4 *hit;     // t, b1, b2, prim (int bits; -1 = miss)
};

struct Shadows {
    float4 *o;   // origin, w: medium (int bits)
    float4 *d;   // target - origin, w: path index (int bits)
    float4 *c;   // contribution before transmittance
    float *w;    // spectral MIS scale applied to L
    int *walk;   // entries whose segment crosses a medium interface (scenes with interfaces)
};

// Device counters of one wavefront: queue lengths, the persistent kernels' work counters, status.
enum {
    kCntActive = 0, kCntNext = 1, kCntShadow = 2, kCntStatus = 3, kCntExtendWork = 4, kCntShadowWork = 5,
    kCntWalk = 6,  // shadow entries queued for the interface walk
    kCntFull = 7,  // paths deferred to the coated / sheen shading pass
    // Batched form: live paths per half of the path slots after the last bounce, and the
    // survivors being counted during the current one.
    kCntLive0 = 8, kCntLive1 = 9, kCntNextLive0 = 10, kCntNextLive1 = 11,
    // Paths filed per shading class by the closest-hit kernel (kClasses entries).
    kCntClass0 = 16,
    kCntSlots = 24
};
enum { kStatusStack = 1, kStatusGuard = 2 };
// Device statistics (64-bit): closest-hit rays, shadow rays, non-empty bounces.
enum { kStatClosest = 0, kStatShadow = 1, kStatBounces = 2, kStatSlots = 4 };

constexpr float kShadowEps = 1e-4f;  // src/scene/interaction.h:21

// Warp-aggregated append: one atomicAdd per warp; returns this thread's slot.
__device__ __forceinline__ int warp_append(int *counter) {
    unsigned mask = __activemask();
    int lane = threadIdx.x & 31;
    int leader = __ffs(mask) - 1;
    int rank = __popc(mask & ((1u << lane) - 1u));
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + rank;
}

// ---------------------------------------------------------------------------------------------
// Pixel filter importance sampling (src/gpu/prender_gpu.cpp:1465-1494; the host builds the CDF
// as src/integrators/gpu_path.cpp:431-456)

static __device__ float filter_eval_1d(const DevScene &s, float x) {
    x = fabsf(x);
    if (x > s.filterRadius) return 0.f;
    switch (s.filterType) {
    case prgpu::FilterGaussian: {
        float is2 = 1.f / (2.f * s.filterSigma * s.filterSigma);
        return fmaxf(0.f, expf(-x * x * is2) - expf(-s.filterRadius * s.filterRadius * is2));
    }
    case prgpu::FilterBlackmanHarris: {
        float t = 0.5f + x / (2.f * s.filterRadius);
        return 0.35875f - 0.48829f * cosf(2.f * kPi * t) + 0.14128f * cosf(4.f * kPi * t) -
               0.01168f * cosf(6.f * kPi * t);
    }
    default: return 1.f;
    }
}

static __device__ float filter_sample_1d(const DevScene &s, float u, float *pdf) {
    int lo = 0, hi = prgpu::kFilterBins;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (__ldg(s.filterCdf + mid) <= u) lo = mid;
        else hi = mid;
    }
    float c0 = __ldg(s.filterCdf + lo), c1 = __ldg(s.filterCdf + lo + 1);
    float w = c1 - c0;
    float t = w > 0.f ? (u - c0) / w : 0.5f;
    float binW = 2.f * s.filterRadius / prgpu::kFilterBins;
    *pdf = w / binW;
    return -s.filterRadius + (float(lo) + t) * binW;
}

// ---------------------------------------------------------------------------------------------
// Surface interaction (src/geometry/shape.cpp:63-85, 224-264)

struct Surf {
    V3 p, n, ns, dpdu;
    float u, v;
};

static __device__ Surf shade_point(const DevScene &s, const prgpu::Primitive &pr, float t, float b1, float b2, V3 o, V3 d) {
    Surf sf;
    if (pr.type == prgpu::PrimSphere) {
        V3 c = f3(pr.p0);
        V3 rel = (o + d * t) - c;
        float l = len(rel);
        V3 n = l > 0.f ? rel * (1.f / l) : mk(0.f, 1.f, 0.f);
        sf.p = c + n * pr.r;
        sf.n = pr.flip ? -n : n;
        sf.ns = sf.n;
        float phi = atan2f(n.z, n.x);
        if (phi < 0.f) phi += 2.f * kPi;
        sf.u = phi * kInv2Pi;
        sf.v = acosf(clampf(n.y, -1.f, 1.f)) * kInvPi;
        sf.dpdu = mk(-rel.z, 0.f, rel.x);
        if (len2(sf.dpdu) < 1e-12f) sf.dpdu = frame_from_z(n).x;
        return sf;
    }
    V3 p0 = f3(pr.p0), p1 = f3(pr.p1), p2 = f3(pr.p2);
    float b0 = 1.f - b1 - b2;
    sf.p = p0 * b0 + p1 * b1 + p2 * b2;
    V3 n = normalize(cross(p1 - p0, p2 - p0));
    sf.u = pr.u0 * b0 + pr.u1 * b1 + pr.u2 * b2;
    sf.v = pr.v0 * b0 + pr.v1 * b1 + pr.v2 * b2;
    V3 ns = n;
    V3 n0 = f3(pr.n0);
    if (len2(n0) > 0.f) {
        ns = n0 * b0 + f3(pr.n1) * b1 + f3(pr.n2) * b2;
        float l = len(ns);
        ns = l > 0.f ? ns * (1.f / l) : n;
        n = face_forward(n, ns);
    }
    sf.n = n;
    sf.ns = ns;
    float du02 = pr.u0 - pr.u2, du12 = pr.u1 - pr.u2, dv02 = pr.v0 - pr.v2, dv12 = pr.v1 - pr.v2;
    float det = du02 * dv12 - dv02 * du12;
    if (fabsf(det) < 1e-9f) {
        sf.dpdu = frame_from_z(n).x;
    } else {
        sf.dpdu = ((p0 - p2) * dv12 - (p1 - p2) * dv02) * (1.f / det);
        if (!isfinite(sf.dpdu.x) || len2(cross(sf.dpdu, n)) == 0.f) sf.dpdu = frame_from_z(n).x;
    }
    return sf;
}

// ---------------------------------------------------------------------------------------------
// Materials (src/materials/material.cpp:73-117; src/gpu/prender_gpu.cpp:1136-1226)

static __device__ Ggx make_ggx(float ax, float ay) {
    Ggx g{ax, ay};
    if (!g.smooth()) {
        g.ax = fmaxf(g.ax, 1e-4f);
        g.ay = fmaxf(g.ay, 1e-4f);
    }
    return g;
}

static __device__ SS diffuse_albedo(const DevScene &s, const prgpu::Material &m, float u, float v, const Lambda &lam) {
    int id = m.albedo;
    if (m.albedoB >= 0 && m.checkerScale > 0.f) {
        int odd = (int(floorf(u * m.checkerScale)) + int(floorf(v * m.checkerScale))) & 1;
        if (odd) id = m.albedoB;
    }
    SS R = tab4(s.spectra, id, lam);
#pragma unroll
    for (int i = 0; i < 4; ++i) R.v[i] = clampf(R.v[i], 0.f, 1.f);
    return R;
}

// Builds the lobe of material m at the hit; may terminate the secondary wavelengths.
static __device__ Lobe make_lobe(const DevScene &s, const prgpu::Material &m, float u, float v, Lambda &lam) {
    Lobe l;
    l.kind = kLobeNone;
    l.etaD = 1.f;
    l.mf = Ggx{0.f, 0.f};
    switch (m.type) {
    case prgpu::MatDiffuse:
        l.kind = kLobeDiffuse;
        l.R = diffuse_albedo(s, m, u, v, lam);
        break;
    case prgpu::MatConductor:
        l.kind = kLobeConductor;
        l.mf = make_ggx(m.alphaX, m.alphaY);
        if (m.eta >= 0) {
            l.eta = tab4(s.spectra, m.eta, lam);
            l.k = tab4(s.spectra, m.k, lam);
        } else {
            // Artist reflectance r -> eta 1, k = 2 sqrt(r) / sqrt(1 - r) (exact r at normal incidence).
            SS r = tab4(s.spectra, m.albedo, lam);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                float ri = clampf(r.v[i], 0.f, 0.9999f);
                l.eta.v[i] = 1.f;
                l.k.v[i] = 2.f * sqrtf(ri) / safe_sqrt(1.f - ri);
            }
        }
        break;
    case prgpu::MatDielectric:
        l.kind = m.thin ? kLobeThin : kLobeDielectric;
        l.etaD = tab(s.spectra, m.eta, lam.l[0]);
        if (m.dispersive) lam.terminate_secondary();
        if (l.etaD == 0.f) l.etaD = 1.f;
        l.mf = make_ggx(m.alphaX, m.alphaY);
        break;
    default: break;
    }
    return l;
}

// make_lobe for a material known to be MatDiffuse (the guided shading class): the lobe kind is a
// constant, so the code of the other kinds drops out of the kernels that use it.
static __device__ __forceinline__ Lobe diffuse_lobe(const DevScene &s, const prgpu::Material &m, float u, float v,
                                                    const Lambda &lam) {
    Lobe l;
    l.kind = kLobeDiffuse;
    l.etaD = 1.f;
    l.mf = Ggx{0.f, 0.f};
    l.R = diffuse_albedo(s, m, u, v, lam);
    return l;
}

// ---------------------------------------------------------------------------------------------
// Image textures (pr::ImageData::Lookup / ImageSpectrumTexture::Evaluate, texture.cpp:8-53) and the
// albedo uplift through the RGB -> spectrum table (RGBToSpectrumTable, rgb2spec.cpp:278-305).

__device__ __forceinline__ int tex_wrap(int v, int n, int mode) {
    if (mode == prgpu::WrapClamp) return min(max(v, 0), n - 1);
    if (mode == prgpu::WrapMirror) {
        int period = 2 * n;
        v %= period;
        if (v < 0) v += period;
        return v < n ? v : period - 1 - v;
    }
    v %= n;
    return v < 0 ? v + n : v;
}

static __device__ void tex_rgb(const DevTex &t, float u, float v, float rgb[3]) {
    u = u * t.su + t.ou;
    v = v * t.sv + t.ov;
    if (t.flipV) v = 1.f - v;
    float x = u * t.w - 0.5f, y = v * t.h - 0.5f;
    int x0 = int(floorf(x)), y0 = int(floorf(y));
    float dx = x - x0, dy = y - y0;
    int xa = tex_wrap(x0, t.w, t.wrap), xb = tex_wrap(x0 + 1, t.w, t.wrap);
    int ya = tex_wrap(y0, t.h, t.wrap), yb = tex_wrap(y0 + 1, t.h, t.wrap);
    const float *a = t.rgb + 3 * (size_t(ya) * t.w + xa), *b = t.rgb + 3 * (size_t(ya) * t.w + xb);
    const float *c = t.rgb + 3 * (size_t(yb) * t.w + xa), *d = t.rgb + 3 * (size_t(yb) * t.w + xb);
    for (int i = 0; i < 3; ++i)
        rgb[i] = ((1.f - dx) * (1.f - dy) * __ldg(a + i) + dx * (1.f - dy) * __ldg(b + i) + (1.f - dx) * dy * __ldg(c + i) +
                  dx * dy * __ldg(d + i)) * t.scale[i];
}

// Sigmoid-polynomial reflectance of an sRGB triple at the 4 wavelengths (RGBAlbedoSpectrum).
static __device__ SS rgb_albedo(const DevScene &s, float r, float g, float b, const Lambda &lam) {
    float rgb[3] = {clampf(r, 0.f, 1.f), clampf(g, 0.f, 1.f), clampf(b, 0.f, 1.f)};
    float c[3];
    if (rgb[0] == rgb[1] && rgb[1] == rgb[2]) {
        const float v = rgb[0], inf = __int_as_float(0x7f800000);
        c[0] = c[1] = 0.f;
        c[2] = v <= 0.f ? -inf : (v >= 1.f ? inf : (v - .5f) / sqrtf(v * (1.f - v)));
    } else {
        const int res = 64;
        int maxc = (rgb[0] > rgb[1]) ? ((rgb[0] > rgb[2]) ? 0 : 2) : ((rgb[1] > rgb[2]) ? 1 : 2);
        float z = rgb[maxc];
        float x = rgb[(maxc + 1) % 3] * (res - 1) / z, y = rgb[(maxc + 2) % 3] * (res - 1) / z;
        int xi = min(int(x), res - 2), yi = min(int(y), res - 2);
        int lo = 0, hi = res - 1;  // largest zi in [0, res - 2] with zNodes[zi] < z
        while (hi - lo > 1) {
            int mid = (lo + hi) >> 1;
            if (__ldg(s.rgbZ + mid) < z) lo = mid;
            else hi = mid;
        }
        int zi = min(lo, res - 2);
        float z0 = __ldg(s.rgbZ + zi), z1 = __ldg(s.rgbZ + zi + 1);
        float dx = x - xi, dy = y - yi, dz = (z - z0) / (z1 - z0);
        auto co = [&](int zz, int yy, int xx, int i) {
            return __ldg(s.rgbCoeffs + 3 * (((size_t(maxc) * res + zz) * res + yy) * res + xx) + i);
        };
        auto lerp = [](float t, float a, float b2) { return (1.f - t) * a + t * b2; };
        for (int i = 0; i < 3; ++i)
            c[i] = lerp(dz, lerp(dy, lerp(dx, co(zi, yi, xi, i), co(zi, yi, xi + 1, i)),
                                 lerp(dx, co(zi, yi + 1, xi, i), co(zi, yi + 1, xi + 1, i))),
                        lerp(dy, lerp(dx, co(zi + 1, yi, xi, i), co(zi + 1, yi, xi + 1, i)),
                             lerp(dx, co(zi + 1, yi + 1, xi, i), co(zi + 1, yi + 1, xi + 1, i))));
    }
    SS out;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float xv = fmaf(lam.l[i], fmaf(lam.l[i], c[0], c[1]), c[2]);
        out.v[i] = isinf(xv) ? (xv > 0.f ? 1.f : 0.f) : 0.5f + xv / (2.f * sqrtf(1.f + xv * xv));
    }
    return out;
}

// ---------------------------------------------------------------------------------------------
// Procedural textures: NoiseFloatTexture (texture.cpp:55-60) over the fBm of noise.cuh, and the
// TextureNode trees.

// Where a texture is evaluated: the hit point and its (u, v).
struct TexCtx {
    V3 p;
    float u, v;
};

static __device__ float noise_node(const prgpu::TextureNode &n, const TexCtx &c) {
    V3 p = (n.flags & prgpu::TexNoiseWorldSpace) ? c.p : mk(c.u, c.v, 0.f);
    p = (p + mk(n.offset[0], n.offset[1], n.offset[2])) * n.frequency;
    const bool turb = (n.flags & prgpu::TexNoiseTurbulence) != 0;
    const float v = fbm_noise(p, n.octaves, turb);
    return turb ? clampf(v * 1.6f, 0.f, 1.f) : clampf(0.5f + 0.5f * v * 1.4f, 0.f, 1.f);
}

// Walks the texture tree under `root` as a weighted sum over its leaves: a checker passes its
// weight to the child its (s, t) cell picks, a mix splits it by its clamped noise. leaf(node, w)
// adds a constant, image or noise leaf. Validated trees are at most 8 deep, so the stack of 10
// never overflows; the guard bounds the walk all the same.
constexpr int kTexStack = 10;
template <class Leaf>
__device__ __forceinline__ void walk_texture(const DevScene &s, int root, const TexCtx &c, Leaf &&leaf) {
    int node[kTexStack];
    float wt[kTexStack];
    node[0] = root;
    wt[0] = 1.f;
    int sp = 1;
    for (int guard = 0; sp > 0 && guard < 64; ++guard) {
        --sp;
        const int id = node[sp];
        const float w = wt[sp];
        const prgpu::TextureNode &n = s.texNodes[id];
        if (n.type == prgpu::TexChecker) {
            const float ss = c.u * n.scaleU + n.offsetU, tt = c.v * n.scaleV + n.offsetV;
            const bool odd = ((int(floorf(ss)) + int(floorf(tt))) & 1) != 0;
            node[sp] = odd ? n.b : n.a;
            wt[sp] = w;
            ++sp;
        } else if (n.type == prgpu::TexMix) {
            if (sp + 2 > kTexStack) continue;
            const float t = clampf(noise_node(s.texNodes[n.t], c), 0.f, 1.f);
            node[sp] = n.a;
            wt[sp] = w * (1.f - t);
            node[sp + 1] = n.b;
            wt[sp + 1] = w * t;
            sp += 2;
        } else {
            leaf(n, w);
        }
    }
}

// A spectrum tree as an albedo at the 4 wavelengths (constants from the spectrum table, images
// uplifted through the RGB -> spectrum table).
static __device__ SS rgb_unbounded(const DevScene &s, float r, float g, float b, const Lambda &lam);

static __device__ SS spectrum_texture(const DevScene &s, int root, const TexCtx &c, const Lambda &lam, bool unbounded = false) {
    SS acc = splat(0.f);
    walk_texture(s, root, c, [&](const prgpu::TextureNode &n, float w) {
        SS v;
        if (n.type == prgpu::TexConstant) {
            v = tab4(s.spectra, n.a, lam);
        } else if (n.type == prgpu::TexImage) {
            float rgb[3];
            tex_rgb(s.textures[n.a], c.u, c.v, rgb);
            v = unbounded ? rgb_unbounded(s, rgb[0], rgb[1], rgb[2], lam) : rgb_albedo(s, rgb[0], rgb[1], rgb[2], lam);
        } else {
            return;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) acc.v[i] += w * v.v[i];
    });
    return acc;
}

static __device__ float float_texture(const DevScene &s, int root, const TexCtx &c) {
    float acc = 0.f;
    walk_texture(s, root, c, [&](const prgpu::TextureNode &n, float w) {
        float v = 0.f;
        if (n.type == prgpu::TexConstant) {
            v = n.value;
        } else if (n.type == prgpu::TexImage) {
            float rgb[3];
            tex_rgb(s.textures[n.a], c.u, c.v, rgb);
            v = n.channel < 0 ? (rgb[0] + rgb[1] + rgb[2]) / 3.f : (n.channel == 0 ? rgb[0] : n.channel == 1 ? rgb[1] : rgb[2]);
        } else if (n.type == prgpu::TexNoise) {
            v = noise_node(n, c);
        }
        acc += w * v;
    });
    return acc;
}

// The textured parameters of material index mi at a hit, applied to its lobe: the reflectance of
// a diffuse lobe (a tree, else an image; clamped to [0, 1] as DiffuseMaterial::GetBxDF,
// material.cpp:73-77) and the roughness of conductor and rough dielectric lobes (trees; alpha =
// clamp(r, 0, 1)^2, material.cpp:80-85, 110-116, 151-154).
static __device__ void textured_lobe(const DevScene &s, int mi, const TexCtx &c, const Lambda &lam, Lobe *l,
                              float etaScale = 1.f) {
    if (!s.matTex) return;
    if (l->kind == kLobeDiffuse) {
        const int tree = s.matTex[5 * mi + 1].w, img = s.matTex[5 * mi].x;
        if (tree >= 0) {
            SS r = spectrum_texture(s, tree, c, lam);
#pragma unroll
            for (int i = 0; i < 4; ++i) r.v[i] = clampf(r.v[i], 0.f, 1.f);
            l->R = r;
        } else if (img >= 0) {
            float rgb[3];
            tex_rgb(s.textures[img], c.u, c.v, rgb);
            l->R = rgb_albedo(s, rgb[0], rgb[1], rgb[2], lam);
        }
    } else if (l->kind == kLobeConductor || l->kind == kLobeDielectric) {
        const int4 m4 = s.matTex[5 * mi + 4];
        if (l->kind == kLobeConductor && m4.x >= 0 && m4.y >= 0) {
            // Divided by the coat's IOR under a coat, as CoatedConductorMaterial (material.cpp:157-158).
            SS e = spectrum_texture(s, m4.x, c, lam, true), k = spectrum_texture(s, m4.y, c, lam, true);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                e.v[i] = e.v[i] / etaScale;
                k.v[i] = k.v[i] / etaScale;
            }
            l->eta = e;
            l->k = k;
        } else if (l->kind == kLobeConductor && s.mats[mi].eta < 0) {
            // A reflectance-parameterised conductor whose reflectance is a texture (tree or image):
            // the artist mapping of make_lobe on the looked-up value, eta 1 and k = 2 sqrt(r) /
            // sqrt(1 - r) with r clamped to [0, 0.9999] (ConductorMaterial::MakeBxDF,
            // material.cpp:90-96; not divided by a coat's IOR, as CoatedConductorMaterial,
            // material.cpp:159-163).
            const int tree = s.matTex[5 * mi + 1].w, img = s.matTex[5 * mi].x;
            if (tree >= 0 || img >= 0) {
                SS r;
                if (tree >= 0) {
                    r = spectrum_texture(s, tree, c, lam);
                } else {
                    float rgb[3];
                    tex_rgb(s.textures[img], c.u, c.v, rgb);
                    r = rgb_albedo(s, rgb[0], rgb[1], rgb[2], lam);
                }
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const float ri = clampf(r.v[i], 0.f, 0.9999f);
                    l->eta.v[i] = 1.f;
                    l->k.v[i] = 2.f * sqrtf(ri) / safe_sqrt(1.f - ri);
                }
            }
        }
        const int4 m2 = s.matTex[5 * mi + 2];
        if (m2.y < 0 && m2.z < 0) return;
        const prgpu::Material &m = s.mats[mi];
        float ax = m.alphaX, ay = m.alphaY;
        if (m2.y >= 0) {
            const float r = clampf(float_texture(s, m2.y, c), 0.f, 1.f);
            ax = r * r;
        }
        if (m2.z >= 0) {
            const float r = clampf(float_texture(s, m2.z, c), 0.f, 1.f);
            ay = r * r;
        }
        l->mf = make_ggx(ax, ay);
    }
}

// RGBUnboundedSpectrum (rgb2spec.cpp:327-335): zero for a colour whose largest component is not
// positive, else the sigmoid polynomial of the colour times 1 / scale, scale = 2 max(r, g, b),
// times that scale (the reference's order of operations, so the same bits).
static __device__ SS rgb_unbounded(const DevScene &s, float r, float g, float b, const Lambda &lam) {
    const float m = fmaxf(0.f, fmaxf(r, fmaxf(g, b)));
    SS v;
    if (m == 0.f) {
#pragma unroll
        for (int i = 0; i < 4; ++i) v.v[i] = 0.f;
        return v;
    }
    const float scale = 2.f * m, inv = 1.f / scale;
    v = rgb_albedo(s, r * inv, g * inv, b * inv, lam);
#pragma unroll
    for (int i = 0; i < 4; ++i) v.v[i] = scale * v.v[i];
    return v;
}

// dp/du and dp/dv of the parameterization at a hit (Sphere / Triangle::Intersect, shape.cpp:75-82,
// 237-251): the sphere's scaled by 2 pi and pi, a coordinate system where they degenerate.
static __device__ void surface_dpduv(const prgpu::Primitive &pr, const Surf &sf, V3 *dpdu, V3 *dpdv) {
    if (pr.type == prgpu::PrimSphere) {
        V3 rel = sf.p - f3(pr.p0);
        float cosT = clampf(rel.y / pr.r, -1.f, 1.f), sinT = safe_sqrt(1.f - cosT * cosT);
        *dpdu = mk(-rel.z, 0.f, rel.x) * (2.f * kPi);
        *dpdv = sinT > 1e-6f ? mk(cosT * rel.x / sinT, -pr.r * sinT, cosT * rel.z / sinT) * kPi : mk(0.f, 0.f, 0.f);
        V3 n = pr.flip ? -sf.n : sf.n;
        if (len2(*dpdu) < 1e-12f || len2(*dpdv) < 1e-12f) {
            Frame f = frame_from_z(n);
            *dpdu = f.x;
            *dpdv = f.y;
        }
        return;
    }
    V3 p0 = f3(pr.p0), p1 = f3(pr.p1), p2 = f3(pr.p2);
    V3 n = normalize(cross(p1 - p0, p2 - p0));
    float du02 = pr.u0 - pr.u2, du12 = pr.u1 - pr.u2, dv02 = pr.v0 - pr.v2, dv12 = pr.v1 - pr.v2;
    float det = du02 * dv12 - dv02 * du12;
    bool degenerate = fabsf(det) < 1e-9f;
    if (!degenerate) {
        float inv = 1.f / det;
        *dpdu = ((p0 - p2) * dv12 - (p1 - p2) * dv02) * inv;
        *dpdv = ((p1 - p2) * du02 - (p0 - p2) * du12) * inv;
        degenerate = len2(cross(*dpdu, n)) == 0.f || !isfinite(dpdu->x) || !isfinite(dpdv->x);
    }
    if (degenerate) {
        Frame f = frame_from_z(n);
        *dpdu = f.x;
        *dpdv = f.y;
    }
}

__device__ __forceinline__ float height_at(const DevTex &t, int channel, float u, float v) {
    float c[3];
    tex_rgb(t, u, v, c);
    return channel < 0 ? (c[0] + c[1] + c[2]) / 3.f : c[channel];
}

// Bump and normal maps of material index mi (Material::PerturbShading, material.cpp:16-60): the
// bump map's finite-difference height gradient tilts dp/du and dp/dv along the shading normal;
// the normal map's colour is a direction in the frame of the shading dp/du and normal (the
// bitangent along dp/dv), scaled in the tangent plane; the result stays in the geometric
// hemisphere and the shading dp/du follows it.
static __device__ void perturb_shading(const DevScene &s, int mi, const prgpu::Primitive &pr, Surf *sf) {
    if (!s.matTex) return;
    const int4 mt = s.matTex[5 * mi], bt = s.matTex[5 * mi + 1];
    const int bumpTree = s.matTex[5 * mi + 2].x;
    if (mt.y < 0 && bt.x < 0 && bumpTree < 0) return;
    V3 dpdu, dpdv;
    surface_dpduv(pr, *sf, &dpdu, &dpdv);
    V3 ns = sf->ns, dpdus = dpdu;
    bool changed = false;
    if (bt.x >= 0 || bumpTree >= 0) {
        // The height at (u, v) and the point moved along dp/du or dp/dv with it.
        auto height = [&](float u, float v, V3 p) {
            return bumpTree >= 0 ? float_texture(s, bumpTree, TexCtx{p, u, v}) : height_at(s.textures[bt.x], bt.y, u, v);
        };
        const float du = 1.f / 2048.f, dv = 1.f / 2048.f, scale = __int_as_float(bt.z);
        float h0 = height(sf->u, sf->v, sf->p);
        float dhdu = (height(sf->u + du, sf->v, sf->p + dpdu * du) - h0) / du * scale;
        float dhdv = (height(sf->u, sf->v + dv, sf->p + dpdv * dv) - h0) / dv * scale;
        V3 bu = dpdu + ns * dhdu, bv = dpdv + ns * dhdv;
        V3 n = cross(bu, bv);
        float l = len(n);
        if (l > 0.f && isfinite(l)) {
            n = n * (1.f / l);
            if (dot(n, ns) < 0.f) n = -n;
            ns = n;
            dpdus = bu;
            changed = true;
        }
    }
    if (mt.y >= 0) {
        float c[3];
        tex_rgb(s.textures[mt.y], sf->u, sf->v, c);
        const float strength = __int_as_float(mt.z);
        V3 t = mk(2.f * c[0] - 1.f, 2.f * c[1] - 1.f, 2.f * c[2] - 1.f);
        t.x *= strength;
        t.y *= mt.w ? -strength : strength;
        Frame f = frame_from_xz(dpdus, ns);
        if (dot(f.y, dpdv) < 0.f) f.y = -f.y;
        V3 n = f.x * t.x + f.y * t.y + f.z * fmaxf(t.z, 1e-3f);
        float l = len(n);
        if (l > 0.f && isfinite(l)) {
            ns = n * (1.f / l);
            changed = true;
        }
    }
    if (!changed) return;
    if (dot(ns, sf->n) < 0.f) ns = -ns;
    sf->ns = ns;
    sf->dpdu = dpdus - ns * dot(dpdus, ns);
}

// True for the materials shaded through FullBsdf: coats and anything with a sheen lobe.
__device__ __forceinline__ bool full_material(const prgpu::Material &m) {
    return m.type == prgpu::MatCoatedDiffuse || m.type == prgpu::MatCoatedConductor ||
           (m.sheenWeight > 0.f && m.sheenColor >= 0);
}

// Builds the coated / sheen BSDF of material m (the reference's CoatedDiffuseMaterial,
// CoatedConductorMaterial and Material::GetBSDF sheen wrapper, material.cpp:5-14, 117-166); may
// terminate the secondary wavelengths (dispersive coat).
static __device__ __noinline__ void make_full(const DevScene &s, const prgpu::Material &m, float u, float v, Lambda &lam,
                                       FullBsdf *b) {
    b->layered = b->sheen = b->black = false;
    if (m.type == prgpu::MatCoatedDiffuse || m.type == prgpu::MatCoatedConductor) {
        float coatEta = tab(s.spectra, m.coatEta, lam.l[0]);
        if (m.coatDispersive) lam.terminate_secondary();
        if (coatEta == 0.f) coatEta = 1.f;
        Layered &L = b->lay;
        b->layered = true;
        L.top.kind = kLobeDielectric;
        L.top.etaD = coatEta;
        L.top.mf = make_ggx(m.coatAlpha, m.coatAlpha);
        L.thickness = fmaxf(m.thickness, 1.17549435e-38f);
        L.g = m.coatG;
        L.albedo = splat(0.f);
        if (m.coatAlbedo >= 0) {
            L.albedo = tab4(s.spectra, m.coatAlbedo, lam);
#pragma unroll
            for (int i = 0; i < 4; ++i) L.albedo.v[i] = fmaxf(0.f, L.albedo.v[i]);
        }
        L.hasAlbedo = nonzero(L.albedo);
        L.maxDepth = m.coatMaxDepth;
        L.nSamples = max(1, m.coatSamples);
        if (m.type == prgpu::MatCoatedDiffuse) {
            L.bottom.kind = kLobeDiffuse;
            L.bottom.R = diffuse_albedo(s, m, u, v, lam);
        } else {
            // The conductor sits under the coat: its n, k are relative to the coat's IOR.
            L.bottom.kind = kLobeConductor;
            L.bottom.etaD = 1.f;
            L.bottom.mf = make_ggx(m.alphaX, m.alphaY);
            if (m.eta >= 0) {
                // Divided (not multiplied by the reciprocal), as material.cpp:157-158.
                SS e = tab4(s.spectra, m.eta, lam), k = tab4(s.spectra, m.k, lam);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    e.v[i] = e.v[i] / coatEta;
                    k.v[i] = k.v[i] / coatEta;
                }
                L.bottom.eta = e;
                L.bottom.k = k;
            } else {
                SS r = tab4(s.spectra, m.albedo, lam);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    float ri = clampf(r.v[i], 0.f, 0.9999f);
                    L.bottom.eta.v[i] = 1.f;
                    L.bottom.k.v[i] = 2.f * sqrtf(ri) / safe_sqrt(1.f - ri);
                }
            }
        }
    } else {
        b->base = make_lobe(s, m, u, v, lam);
        b->black = b->base.kind == kLobeNone;
    }
    if (!b->black && m.sheenWeight > 0.f && m.sheenColor >= 0 && s.sheenTable) {
        Sheen &sh = b->sh;
        b->sheen = true;
        sh.color = tab4(s.spectra, m.sheenColor, lam);
#pragma unroll
        for (int i = 0; i < 4; ++i) sh.color.v[i] = fmaxf(0.f, sh.color.v[i]);
        sh.alpha = clampf(m.sheenRoughness, 0.05f, 1.f);
        sh.weight = clampf(m.sheenWeight, 0.f, 1.f);
        sh.colorMax = clampf(max_c(sh.color), 0.f, 1.f);
        sh.table = s.sheenTable;
    }
}

// The textured parameters of a coated / sheen BSDF: its base lobe (textured_lobe), the coat's
// roughness, thickness and medium albedo (MakeCoatTop, material.cpp:119-130) and the sheen's colour
// and roughness (Material::GetBSDF, material.cpp:5-14; SheenBxDF clamps, bxdf.cpp:568-571).
static __device__ void textured_full(const DevScene &s, int mi, const TexCtx &c, const Lambda &lam, FullBsdf *b) {
    if (!s.matTex || b->black) return;
    // A coated conductor's n, k are relative to the coat's IOR.
    textured_lobe(s, mi, c, lam, b->layered ? &b->lay.bottom : &b->base, b->layered ? b->lay.top.etaD : 1.f);
    const int4 m2 = s.matTex[5 * mi + 2], m3 = s.matTex[5 * mi + 3];
    if (b->layered) {
        Layered &L = b->lay;
        if (m3.x >= 0) {
            const float r = clampf(float_texture(s, m3.x, c), 0.f, 1.f);
            L.top.mf = make_ggx(r * r, r * r);
        }
        if (m3.y >= 0) L.thickness = fmaxf(float_texture(s, m3.y, c), 1.17549435e-38f);
        if (m3.z >= 0) {
            L.albedo = spectrum_texture(s, m3.z, c, lam);
#pragma unroll
            for (int i = 0; i < 4; ++i) L.albedo.v[i] = fmaxf(0.f, L.albedo.v[i]);
            L.hasAlbedo = nonzero(L.albedo);
        }
    }
    if (b->sheen) {
        Sheen &sh = b->sh;
        if (m3.w >= 0) {
            sh.color = spectrum_texture(s, m3.w, c, lam);
#pragma unroll
            for (int i = 0; i < 4; ++i) sh.color.v[i] = fmaxf(0.f, sh.color.v[i]);
            sh.colorMax = clampf(max_c(sh.color), 0.f, 1.f);
        }
        if (m2.w >= 0) sh.alpha = clampf(float_texture(s, m2.w, c), 0.05f, 1.f);
    }
}

// ---------------------------------------------------------------------------------------------
// Lights

static __device__ SS emitted(const DevScene &s, const prgpu::Light &l, V3 n, V3 w, const Lambda &lam) {
    float c = dot(n, w);
    if (!l.twoSided && c <= 0.f) return splat(0.f);
    float prof = l.cosPower > 0.f ? powf(fabsf(c), l.cosPower) : 1.f;
    return tab4(s.spectra, l.spectrum, lam) * (l.scale * prof);
}

// Solid-angle density of sampling point p (normal n) on area light l from ref (uniform area).
static __device__ float area_pdf(const prgpu::Light &l, V3 ref, V3 p, V3 n) {
    V3 d = p - ref;
    float d2 = len2(d);
    float c = fabsf(dot(n, d * rsqrtf(d2)));
    if (c == 0.f) return 0.f;
    return d2 / (c * l.area);
}

// Probability that NEE at (p, n) picks light li: the light-BVH pmf when the scene has one (the
// exact leaf-to-root walk), the power pmf otherwise.
static __device__ float light_pmf(const DevScene &s, int li, V3 p, V3 n) {
    if (s.lbvhCount == 0) return s.lights[li].pmf;
    return lbvh_pmf(LightTree{s.lbvh, s.lbvhCount, s.lbvhProb, s.lightLeaf}, li, p, n);
}

// ---------------------------------------------------------------------------------------------
// Image environment and sun (src/lights/light.cpp:217-297, src/lights/sky.cpp:84-109)

// Equirectangular mapping with +y up (light.h:287-297) and the map's rotation about +y.
__device__ __forceinline__ V3 env_to_world(const DevEnvMap &m, V3 v) {
    return mk(m.rc * v.x + m.rs * v.z, v.y, -m.rs * v.x + m.rc * v.z);
}
__device__ __forceinline__ V3 env_to_light(const DevEnvMap &m, V3 v) {
    return mk(m.rc * v.x - m.rs * v.z, v.y, m.rs * v.x + m.rc * v.z);
}
__device__ __forceinline__ void dir_to_equirect(V3 d, float *u, float *v) {
    float theta = acosf(clampf(d.y, -1.f, 1.f));
    float phi = atan2f(d.z, d.x);
    if (phi < 0.f) phi += 2.f * kPi;
    *u = phi * kInv2Pi;
    *v = theta * kInvPi;
}

__device__ __forceinline__ float texel_at(const float4 &t, float l) {
    float x = fmaf(l, fmaf(l, t.x, t.y), t.z);
    float sg = isinf(x) ? (x > 0.f ? 1.f : 0.f) : 0.5f + x / (2.f * sqrtf(1.f + x * x));
    return t.w * sg;
}

// Radiance of the map towards world direction d: bilinear texel spectra with horizontal wrap
// (EnvironmentLight::Lookup, light.cpp:238-261), times the illuminant and the scale.
static __device__ SS env_lookup(const DevScene &s, V3 d, const Lambda &lam) {
    const DevEnvMap &m = s.envMap;
    float u, v;
    dir_to_equirect(normalize(env_to_light(m, d)), &u, &v);
    float x = u * m.w - 0.5f, y = v * m.h - 0.5f;
    int x0 = int(floorf(x)), y0 = int(floorf(y));
    float dx = x - x0, dy = y - y0;
    SS r = splat(0.f);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        int xi = x0 + (k & 1), yi = y0 + (k >> 1);
        xi = ((xi % m.w) + m.w) % m.w;
        yi = min(max(yi, 0), m.h - 1);
        float wgt = ((k & 1) ? dx : 1.f - dx) * ((k >> 1) ? dy : 1.f - dy);
        float4 t = __ldg(m.texels + size_t(yi) * m.w + xi);
#pragma unroll
        for (int i = 0; i < 4; ++i) r.v[i] += wgt * texel_at(t, lam.l[i]);
    }
    if (m.illuminant >= 0) r = r * tab4(s.spectra, m.illuminant, lam);
    return r * m.scale;
}

// Distribution1D::SampleContinuous over a CDF of n + 1 entries (sampling.cpp).
__device__ __forceinline__ float dist1d_sample(const float *cdf, int n, float u, int *off) {
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (__ldg(cdf + mid) <= u) lo = mid;
        else hi = mid;
    }
    float c0 = __ldg(cdf + lo), c1 = __ldg(cdf + lo + 1);
    float du = u - c0;
    if (c1 - c0 > 0.f) du /= c1 - c0;
    *off = lo;
    return (float(lo) + du) / float(n);
}

// Direction and solid-angle pdf from the map's 2D distribution (EnvironmentLight::SampleLi).
static __device__ bool env_sample(const DevScene &s, float u0, float u1, V3 *wi, float *pdf) {
    const DevEnvMap &m = s.envMap;
    if (!(m.margInt > 0.f)) return false;
    int iv, iu;
    float v = dist1d_sample(m.margCdf, m.h, u1, &iv);
    float u = dist1d_sample(m.rowCdf + size_t(iv) * (m.w + 1), m.w, u0, &iu);
    float rowInt = __ldg(m.rowInt + iv);
    if (!(rowInt > 0.f)) return false;
    float mapPdf = (__ldg(m.func + size_t(iv) * m.w + iu) / rowInt) * (rowInt / m.margInt);
    float theta = v * kPi, phi = u * 2.f * kPi;
    float st = sinf(theta);
    if (!(st > 0.f) || !(mapPdf > 0.f)) return false;
    *wi = env_to_world(m, mk(st * cosf(phi), cosf(theta), st * sinf(phi)));
    *pdf = mapPdf / (2.f * kPi * kPi * st);
    return true;
}

// Solid-angle pdf of sampling world direction d (EnvironmentLight::PDF_Li).
static __device__ float env_pdf(const DevScene &s, V3 d) {
    const DevEnvMap &m = s.envMap;
    if (!(m.margInt > 0.f)) return 0.f;
    float u, v;
    dir_to_equirect(normalize(env_to_light(m, d)), &u, &v);
    float st = sinf(v * kPi);
    if (!(st > 0.f)) return 0.f;
    int iu = min(max(int(u * m.w), 0), m.w - 1), iv = min(max(int(v * m.h), 0), m.h - 1);
    return __ldg(m.func + size_t(iv) * m.w + iu) / m.margInt / (2.f * kPi * kPi * st);
}

__device__ __forceinline__ float sun_pdf(const DevSun &u) { return 1.f / (2.f * kPi * (1.f - u.cosMax)); }

struct LightSample {
    V3 wi, target;
    SS Le;
    float pdf;   // selection pmf times the solid-angle density (1 for point lights)
    bool delta;
    bool ok;
};

// Chooses a light and a point on it as seen from p (normal n, zero in media).
// SmoothStep(x, a, b) of the reference's math (a == b: a step at a).
__device__ __forceinline__ float smooth_step(float x, float a, float b) {
    if (a == b) return x < a ? 0.f : 1.f;
    float t = clampf((x - a) / (b - a), 0.f, 1.f);
    return t * t * (3.f - 2.f * t);
}

// Largest i in [0, n - 2] with v[i] <= x (FindInterval over a sorted table).
__device__ __forceinline__ int find_interval(const float *v, int n, float x) {
    int lo = 0, hi = n - 1;
    if (!(__ldg(v) <= x)) return 0;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (__ldg(v + mid) <= x) lo = mid;
        else hi = mid;
    }
    return min(lo, n - 2);
}

// Relative intensity of a type C IES profile towards the profile-frame direction w
// (IESProfile::Evaluate / EvaluateAngles, ies.cpp:79-109): theta from the nadir axis, phi folded
// by the symmetry the last horizontal angle implies, then linear in theta and in phi.
static __device__ float ies_eval(const DevDelta &l, V3 w) {
    const float *va = l.profile, *ha = l.profile + l.nV, *cd = l.profile + l.nV + l.nH;
    const float deg = 57.295779513082320876f;
    float theta = acosf(clampf(w.z, -1.f, 1.f)) * deg;
    float phi = atan2f(w.y, w.x) * deg;
    const int nV = l.nV, nH = l.nH;
    if (theta < __ldg(va) || theta > __ldg(va + nV - 1)) return 0.f;
    float hLast = __ldg(ha + nH - 1);
    phi = fmodf(phi, 360.f);
    if (phi < 0.f) phi += 360.f;
    if (nH == 1 || hLast == 0.f) {
        phi = 0.f;
    } else if (hLast <= 90.f) {
        phi = fmodf(phi, 180.f);
        if (phi > 90.f) phi = 180.f - phi;
    } else if (hLast <= 180.f) {
        if (phi > 180.f) phi = 360.f - phi;
    }
    auto lookupV = [&](int hi) {
        if (nV == 1) return __ldg(cd + size_t(hi) * nV);
        int vi = find_interval(va, nV, theta);
        float t = (theta - __ldg(va + vi)) / fmaxf(1e-6f, __ldg(va + vi + 1) - __ldg(va + vi));
        t = clampf(t, 0.f, 1.f);
        float a0 = __ldg(cd + size_t(hi) * nV + vi), a1 = __ldg(cd + size_t(hi) * nV + vi + 1);
        return (1.f - t) * a0 + t * a1;
    };
    if (nH == 1) return lookupV(0);
    int hi = find_interval(ha, nH, phi);
    float t = clampf((phi - __ldg(ha + hi)) / fmaxf(1e-6f, __ldg(ha + hi + 1) - __ldg(ha + hi)), 0.f, 1.f);
    return (1.f - t) * lookupV(hi) + t * lookupV(hi + 1);
}

// A spot, distant or goniometric light's sample towards p (delta distributions: pdf = the
// selection pmf).
__device__ __forceinline__ LightSample sample_delta_light(const DevScene &s, const DevDelta &l, V3 p, const Lambda &lam) {
    LightSample ls;
    ls.ok = false;
    ls.delta = true;
    ls.pdf = l.pmf;
    if (l.type == prgpu::DeltaDistant) {  // DistantLight::SampleLi, sky.cpp:52-61
        ls.wi = l.dir;
        ls.target = p + l.dir * (2.f * s.worldRadius);
        ls.Le = tab4(s.spectra, l.spectrum, lam) * l.scale;
    } else {
        V3 dd = l.pos - p;
        float d2 = len2(dd);
        if (!(d2 > 0.f)) return ls;
        ls.wi = dd * rsqrtf(d2);
        float f;
        if (l.type == prgpu::DeltaSpot) {  // SpotLight::SampleLi, light.cpp:168-192
            f = smooth_step(dot(-ls.wi, l.dir), l.cosEnd, l.cosStart);
        } else {  // GoniometricLight::SampleLi, sky.cpp:12-26
            V3 w = -ls.wi;
            f = ies_eval(l, mk(dot(w, l.fx), dot(w, l.fy), dot(w, l.fz)));
        }
        if (!(f > 0.f)) return ls;
        ls.target = l.pos;
        ls.Le = tab4(s.spectra, l.spectrum, lam) * (l.scale * f / d2);
    }
    ls.ok = ls.pdf > 0.f;
    return ls;
}

static __device__ LightSample sample_light(const DevScene &s, V3 p, V3 n, const Lambda &lam, float ul, float u0, float u1) {
    LightSample ls;
    ls.ok = false;
    ls.delta = false;
    // Infinite lights first: constant environment, image environment, sun, each with its pmf.
    float acc = 0.f;
    if (s.envSpectrum >= 0) {
        if (ul < s.envPmf) {
            float z = 1.f - 2.f * u0, r = safe_sqrt(1.f - z * z), sp, cp;
            sincosf(2.f * kPi * u1, &sp, &cp);
            ls.wi = mk(r * cp, r * sp, z);
            ls.target = p + ls.wi * (2.f * s.worldRadius);
            ls.Le = tab4(s.spectra, s.envSpectrum, lam) * s.envScale;
            ls.pdf = s.envPmf * kInv4Pi;
            ls.ok = true;
            return ls;
        }
        acc = s.envPmf;
    }
    if (s.envMap.w > 0) {
        if (ul < acc + s.envMap.pmf) {
            float pdf;
            if (!env_sample(s, u0, u1, &ls.wi, &pdf)) return ls;
            ls.target = p + ls.wi * (2.f * s.worldRadius);
            ls.Le = env_lookup(s, ls.wi, lam);
            ls.pdf = s.envMap.pmf * pdf;
            ls.ok = nonzero(ls.Le) && ls.pdf > 0.f;
            return ls;
        }
        acc += s.envMap.pmf;
    }
    if (s.sun.spectrum >= 0) {
        if (ul < acc + s.sun.pmf) {
            // SampleUniformCone (sampling.h): cos theta = (1 - u0) + u0 cos theta_max.
            float ct = (1.f - u0) + u0 * s.sun.cosMax, st = safe_sqrt(1.f - ct * ct), sp, cp;
            sincosf(2.f * kPi * u1, &sp, &cp);
            ls.wi = s.sun.x * (st * cp) + s.sun.y * (st * sp) + s.sun.z * ct;
            ls.target = p + ls.wi * (2.f * s.worldRadius);
            ls.Le = tab4(s.spectra, s.sun.spectrum, lam) * s.sun.scale;
            ls.pdf = s.sun.pmf * sun_pdf(s.sun);
            ls.ok = true;
            return ls;
        }
        acc += s.sun.pmf;
    }
    int li = -1;
    float pmf = 0.f;
    if (s.lbvhCount > 0) {
        float u = fminf((ul - acc) / s.lbvhProb, kOneMinusEps);
        li = lbvh_sample(LightTree{s.lbvh, s.lbvhCount, s.lbvhProb, s.lightLeaf}, p, n, u, &pmf);
    } else {
        if (s.lightCount == 0) return ls;
        li = s.lightCount - 1;
        for (int i = 0; i < s.lightCount; ++i) {
            acc += s.lights[i].pmf;
            if (ul < acc) {
                li = i;
                break;
            }
        }
        pmf = s.lights[li].pmf;
    }
    if (li < 0 || !(pmf > 0.f)) return ls;
    const prgpu::Light &l = s.lights[li];
    if (l.type == prgpu::LightPoint) {
        ls.target = f3(l.position);
        V3 dd = ls.target - p;
        float d2 = len2(dd);
        if (!(d2 > 0.f)) return ls;
        ls.wi = dd * rsqrtf(d2);
        ls.Le = tab4(s.spectra, l.spectrum, lam) * (l.scale / d2);
        ls.pdf = pmf;
        ls.delta = true;
        ls.ok = true;
        return ls;
    }
    const prgpu::Primitive &lp = s.prims[l.primitive];
    V3 pl, nl;
    if (lp.type == prgpu::PrimSphere) {
        float z = 1.f - 2.f * u0, r = safe_sqrt(1.f - z * z), sp, cp;
        sincosf(2.f * kPi * u1, &sp, &cp);
        V3 nn = mk(r * cp, r * sp, z);
        pl = f3(lp.p0) + nn * lp.r;
        nl = lp.flip ? -nn : nn;
    } else {
        float b0, b1;
        if (u0 < u1) {
            b0 = u0 * 0.5f;
            b1 = u1 - b0;
        } else {
            b1 = u1 * 0.5f;
            b0 = u0 - b1;
        }
        float b2 = 1.f - b0 - b1;
        V3 p0 = f3(lp.p0), p1 = f3(lp.p1), p2 = f3(lp.p2);
        pl = p0 * b0 + p1 * b1 + p2 * b2;
        nl = normalize(cross(p1 - p0, p2 - p0));
        V3 n0 = f3(lp.n0);
        if (len2(n0) > 0.f) nl = face_forward(nl, n0 * b0 + f3(lp.n1) * b1 + f3(lp.n2) * b2);
    }
    V3 dd = pl - p;
    float d2 = len2(dd);
    if (!(d2 > 0.f)) return ls;
    ls.wi = dd * rsqrtf(d2);
    ls.Le = emitted(s, l, nl, -ls.wi, lam);
    ls.pdf = pmf * area_pdf(l, p, pl, nl);
    if (!nonzero(ls.Le) || !(ls.pdf > 0.f) || !isfinite(ls.pdf)) return ls;
    ls.target = pl + (dot(-dd, nl) < 0.f ? -nl : nl) * ray_eps(pl);
    ls.ok = true;
    return ls;
}

// Transmittance of the shadow segment o -> o + dd (length len(dd)) in the given medium.
static __device__ SS segment_tr(const DevScene &s, int medium, const Lambda &lam, V3 o, V3 dd, float frac) {
    float l = len(dd);
    float dist = frac * l;
    if (!is_grid(s, medium)) return homogeneous_tr(s, medium, lam, dist);
    Pcg rng = segment_stream(o, dd, uint32_t(medium));
    return medium_transmittance(s, medium, lam, o, dd * (1.f / l), dist, rng);
}

// ---------------------------------------------------------------------------------------------
// Kernels

struct ChunkInfo {
    int pixBegin;      // first pixel of the chunk (raster index)
    int npix;          // pixels in the chunk
    int samples;       // samples per pixel in the chunk
    int firstSample;   // absolute sample index of the chunk's first sample
    uint64_t seed;
    int maxDepth;      // <= 0: unlimited
};

__device__ __forceinline__ Lambda load_lam(const Paths &P, int j) {
    float4 a = P.lam[j], b = P.lpdf[j];
    Lambda w;
    w.l[0] = a.x; w.l[1] = a.y; w.l[2] = a.z; w.l[3] = a.w;
    w.pdf[0] = b.x; w.pdf[1] = b.y; w.pdf[2] = b.z; w.pdf[3] = b.w;
    return w;
}

// Render index of a path, kept in bits 24..31 of meta.w (0 outside batches).
constexpr int kRenderShift = 24;
__device__ __forceinline__ int path_render(int metaw) { return int(unsigned(metaw) >> kRenderShift); }

// The scene of a path: the kernel argument for single renders, the batch table otherwise (kept
// apart so the single-render form reads its scene from the parameter space).
template <bool kBatch> struct SceneOf;
template <> struct SceneOf<false> {
    static __device__ __forceinline__ const DevScene &get(const DevScene &s0, const DevScene *, int) { return s0; }
};
template <> struct SceneOf<true> {
    static __device__ __forceinline__ const DevScene &get(const DevScene &, const DevScene *t, int rid) { return t[rid]; }
};

// Camera sample `sample` of pixel `pix` (PerspectiveCamera::GenerateRay, camera.cpp:36-48, with
// SampleVisible wavelengths and filter importance sampling) into path slot j, queued if valid.
// Camera ray through film position (fx, fy) with lens sample (l0, l1) (PerspectiveCamera::
// GenerateRay, camera.cpp:36-48): world origin and unit direction.
__device__ __forceinline__ void camera_ray(const DevScene &s, float fx, float fy, float l0, float l1, V3 *o, V3 *d) {
    const prgpu::Camera &c = s.cam;
    V3 dir = normalize(mk((2.f * fx / c.width - 1.f) * c.tanHalfFov * c.aspect, (1.f - 2.f * fy / c.height) * c.tanHalfFov, 1.f));
    V3 org = mk(0.f, 0.f, 0.f);
    if (c.lensRadius > 0.f) {
        float lx, ly;
        concentric_disk(l0, l1, &lx, &ly);
        V3 pf = dir * (c.focalDistance / dir.z);
        org = mk(lx * c.lensRadius, ly * c.lensRadius, 0.f);
        dir = normalize(pf - org);
    }
    const float *M = c.cameraToWorld;
    *o = mk(M[0] * org.x + M[1] * org.y + M[2] * org.z + M[3], M[4] * org.x + M[5] * org.y + M[6] * org.z + M[7],
            M[8] * org.x + M[9] * org.y + M[10] * org.z + M[11]);
    *d = normalize(mk(M[0] * dir.x + M[1] * dir.y + M[2] * dir.z, M[4] * dir.x + M[5] * dir.y + M[6] * dir.z,
                      M[8] * dir.x + M[9] * dir.y + M[10] * dir.z));
}

__device__ __forceinline__ void raygen_path(const DevScene &s, const Paths &P, int j, int pix, uint64_t sample,
                                            uint64_t seed, int rid, int *counters, int *queue) {
    {
        int px = pix % s.cam.width, py = pix / s.cam.width;
        Pcg rng = pixel_sample_stream(uint32_t(pix), sample, seed);
        Lambda lam = sample_visible(rng.uniform());
        float pdfX, pdfY;
        float dx = filter_sample_1d(s, rng.uniform(), &pdfX), dy = filter_sample_1d(s, rng.uniform(), &pdfY);
        float fw = filter_eval_1d(s, dx) * filter_eval_1d(s, dy) * s.filterNorm / (pdfX * pdfY);
        float l0 = rng.uniform(), l1 = rng.uniform();
        V3 o, dw;
        camera_ray(s, float(px) + 0.5f + dx, float(py) + 0.5f + dy, l0, l1, &o, &dw);
        bool valid = fw != 0.f && isfinite(fw);
        P.o[j] = make_float4(o.x, o.y, o.z, 1.f);
        P.d[j] = make_float4(dw.x, dw.y, dw.z, 1.f);
        P.beta[j] = make_float4(1.f, 1.f, 1.f, 1.f);
        P.rpath[j] = make_float4(1.f, 1.f, 1.f, 1.f);
        P.L[j] = make_float4(0.f, 0.f, 0.f, 0.f);
        P.Lhero[j] = make_float4(0.f, 0.f, 0.f, 0.f);
        P.lam[j] = make_float4(lam.l[0], lam.l[1], lam.l[2], lam.l[3]);
        P.lpdf[j] = make_float4(lam.pdf[0], lam.pdf[1], lam.pdf[2], lam.pdf[3]);
        P.rng[j] = make_ulonglong2(rng.state, rng.inc);
        P.meta[j] = make_int4(pix, 0, s.cameraMedium, rid << kRenderShift);
        P.prevP[j] = make_float4(o.x, o.y, o.z, valid ? fw : 0.f);
        P.prevN[j] = make_float4(0.f, 0.f, 0.f, __int_as_float(0));
        if (valid) queue[warp_append(counters + kCntActive)] = j;
    }
}

static __global__ void __launch_bounds__(256) k_raygen(DevScene s, Paths P, ChunkInfo ci, int *counters, int *queue) {
    int total = ci.npix * ci.samples;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < total; j += gridDim.x * blockDim.x) {
        int sIdx = j / ci.npix, pl = j - sIdx * ci.npix;
        raygen_path(s, P, j, ci.pixBegin + pl, uint64_t(ci.firstSample) + uint64_t(sIdx), ci.seed, 0, counters, queue);
    }
}

// Material sort: files every queued path under its shading class (ShadeClass), 256 paths per block
// step: ranks from shared-memory counters, one global atomic per class and block for the block's
// slots, so the shading kernel can walk the classes in order. The order within a class does not
// matter: every path's update depends on its own state only.
template <bool kBatch = false>
// guideMode (single renders; batched renders read their scene's flags): diffuse vertices before a
// path's kGuideVertices-th diffuse vertex are filed as kClassGuided when the render uses the guide.
__global__ void __launch_bounds__(256) k_classify(DevScene s0, const DevScene *scenes, Paths P, int *counters,
                                                  const int *queue, int *classQ, int classCap, int guideMode = 0) {
    __shared__ int hist[kClasses], base[kClasses];
    const int n = counters[kCntActive];
    for (int q0 = blockIdx.x * blockDim.x; q0 < n; q0 += gridDim.x * blockDim.x) {
        if (threadIdx.x < kClasses) hist[threadIdx.x] = 0;
        __syncthreads();
        const int q = q0 + threadIdx.x;
        int c = -1, j = 0, rank = 0;
        if (q < n) {
            j = queue[q];
            const int4 mt = P.meta[j];
            const int prim = __float_as_int(P.hit[j].w);
            const DevScene &s = SceneOf<kBatch>::get(s0, scenes, path_render(mt.w));
            c = mt.z >= 0 ? kClassMedium : (prim < 0 ? kClassMiss : int(__ldg(s.primClass + prim) & ~kTransparentBit));
            const int gm = kBatch ? s.guideMode : guideMode;
            if (c == kClassDiffuse && (gm & 3) && ((mt.w >> 2) & 7) < kGuideVertices) c = kClassGuided;
            rank = atomicAdd(&hist[c], 1);
        }
        __syncthreads();
        if (threadIdx.x < kClasses)
            base[threadIdx.x] = hist[threadIdx.x] ? atomicAdd(counters + kCntClass0 + threadIdx.x, hist[threadIdx.x]) : 0;
        __syncthreads();
        if (c >= 0) classQ[size_t(c) * classCap + base[c] + rank] = j;
        __syncthreads();
    }
}

// Closest hit for every queued path, by persistent warps whose idle lanes take the next queue
// entries (see k_trace_persist in accel.cu): bounce rays are incoherent and end after very
// different numbers of steps. A finished lane's hit is stored when it takes its next entry.
template <bool kSpheres, bool kBatch = false>
// 4 resident blocks (64 registers) for triangle scenes; the batched form would otherwise take 74
// registers and 3 blocks. Scenes with spheres keep the double-precision sphere test unconstrained.
__global__ void __launch_bounds__(256, kSpheres ? 1 : 4) k_extend(DevScene s0, const DevScene *scenes, Paths P,
                                                                  int *counters, const int *queue) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int n = counters[kCntActive];
    __shared__ int2 shortStack[kShortStack * 256];
    HybridStack<kShortStack, 256> hs;
    hs.sh = shortStack + threadIdx.x;
    TraceRay r;
    TravState st;
    st.ref = 0;
    st.sp = 0;
    st.tMax = kInf;
    st.found = false;
    st.hit.prim = -1;
    int j = 0;
    const QNode *nodes = s0.qnodes;
    const LeafPrim *leaves = s0.leaves;
    bool active = false, exhausted = n == 0, pending = false, overflow = false;
    while (!__all_sync(full, exhausted)) {
        const bool idle = !active && !exhausted;
        const unsigned need = __ballot_sync(full, idle), busy = __ballot_sync(full, active);
        if (need && (__popc(need) >= kRefillLanes || !busy)) {
            int base = 0;
            if (lane == 0) base = atomicAdd(counters + kCntExtendWork, __popc(need));
            base = __shfl_sync(full, base, 0);
            if (idle) {
                if (pending) {
                    const Hit h = finish_hit<kSpheres>(leaves, r, st);
                    P.hit[j] = make_float4(h.t, h.u, h.v, __int_as_float(h.prim));
                }
                pending = false;
                int q = base + __popc(need & ((1u << lane) - 1u));
                if (q >= n) {
                    exhausted = true;
                } else {
                    j = queue[q];
                    const DevScene &s = SceneOf<kBatch>::get(s0, scenes, path_render(P.meta[j].w));
                    nodes = s.qnodes;
                    leaves = s.leaves;
                    float4 o = P.o[j], d = P.d[j];
                    r = make_trace_ray(mk(o.x, o.y, o.z), mk(d.x, d.y, d.z));
                    st.tMax = kInf;
                    st.sp = 0;
                    st.found = false;
                    st.hit = Hit{0.f, 0.f, 0.f, -1};
                    float te;
                    active = !s.root.empty &&
                             box_entry(r, s.root.box[0], s.root.box[1], s.root.box[2], s.root.box[3], s.root.box[4],
                                       s.root.box[5], &te) &&
                             te < kInf;
                    st.ref = s.root.ref;
                    // A ray that misses the root: a miss (t, u, v 0), stored at the next refill.
                    pending = !active;
                }
            }
        }
        if (active && traverse4_step_st<false, kSpheres, false, true>(nodes, leaves, r, st, hs, &overflow)) {
            active = false;
            pending = true;
        }
    }
    if (overflow) atomicOr(counters + kCntStatus, kStatusStack);
}

struct ShadeArgs {
    DevScene s;
    const DevScene *scenes;  // the renders' scenes in device memory (batched form: by path_render)
    Paths P;
    Shadows S;
    const int *classQ;       // the closest-hit kernel's per-class queues (kClasses x classCap)
    int classCap;
    int *queueOut;
    int *counters;
    int maxDepth;
    int halfSlots;           // batched form: slots [0, halfSlots) are half 0, the rest half 1
    // Guided form: network outputs by position in the diffuse class queue, the per-path training
    // records (kGuideVertices of 4 float4 each: xn + mean beta, n + BSDF pdf, wo + radiance
    // snapshot, wi + state), and the mode (bit 0 sample with the guide, bit 1 record samples).
    const float *guideOut;
    float4 *guideRec;
    int guideMode;
    // Paths that reached a coated / sheen surface, deferred by the main pass to the kFull pass
    // (the ping-pong queue being consumed, free while shading runs).
    int *fullQ;
    GuideOpts guideOpts;     // guided form: the decoding settings of the network outputs
};

// One bounce of PathIntegrator::Li for every active path (path.cpp:155-236). The main pass
// (kFull = false) defers paths that reach a coated or sheen surface, after their free flight and
// emission, to the fullQ queue; the kFull pass shades those surfaces. Keeping the layered code out
// of the main pass keeps its register allocation that of the plain materials. kDelta: the scene has
// spot / distant / goniometric lights or image textures (their code is instantiated only then).
// kGuide: this launch shades the guided class (kClassGuided) only, sampling with the guide; the
// main pass (kGuide false) shades every other class, so the plain materials keep the plain code.
template <bool kBatch = false, bool kGuide = false, bool kFull = false, bool kDelta = false>
__global__ void __launch_bounds__(256, 2) k_shade(ShadeArgs a) {
    const Paths &P = a.P;
    // The classes laid end to end: entry q belongs to the class whose prefix range holds it.
    int start[kClasses + 1];
    start[0] = 0;
#pragma unroll
    for (int c = 0; c < kClasses; ++c) start[c + 1] = start[c] + a.counters[kCntClass0 + c];
    const int q0 = kGuide ? start[kClassGuided] : 0;
    const int n = kFull ? a.counters[kCntFull] : (kGuide ? start[kClasses] : start[kClassGuided]);
    for (int q = q0 + blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        int c = kFull ? int(kClassOther) : (kGuide ? int(kClassGuided) : 0);
        int first = kGuide ? q0 : 0;
        if constexpr (!kFull && !kGuide) {
#pragma unroll
            for (int k = 1; k < kClassGuided; ++k)
                if (q >= start[k]) {
                    c = k;
                    first = start[k];
                }
        }
        int j = kFull ? a.fullQ[q] : a.classQ[size_t(c) * a.classCap + (q - first)];
        int4 meta = P.meta[j];
        const DevScene &s = a.scenes[kBatch ? path_render(meta.w) : 0];
        const int maxDepth = kBatch ? s.maxDepth : a.maxDepth;
        float4 o4 = P.o[j], d4 = P.d[j], hit = P.hit[j];
        V3 o = mk(o4.x, o4.y, o4.z), d = mk(d4.x, d4.y, d4.z);
        float prevPdf = o4.w, etaScale = d4.w;
        SS beta = from_f4(P.beta[j]), rpath = from_f4(P.rpath[j]);
        SS L = from_f4(P.L[j]), Lhero = from_f4(P.Lhero[j]);
        Lambda lam = load_lam(P, j);
        ulonglong2 rs = P.rng[j];
        Pcg rng{rs.x, rs.y};
        int depth = meta.y, medium = meta.z, flags = meta.w;
        bool specular = flags & 1;
        int gcount = (flags >> 2) & 7;  // guided form: diffuse vertices passed (capped at kGuideVertices)
        int crossings = (flags >> 8) & 0xffff;
        float4 pp4 = P.prevP[j], pn4 = P.prevN[j];
        V3 prevP = mk(pp4.x, pp4.y, pp4.z), prevN = mk(pn4.x, pn4.y, pn4.z);
        int iters = __float_as_int(pn4.w) + (kFull ? 0 : 1);
        int prim = __float_as_int(hit.w);
        bool alive = true, deferred = false;
        // Guide mode of this path: the call's, restricted in the batched form to its render's flags.
        const int gmode = kBatch ? (a.guideMode & s.guideMode) : a.guideMode;
        if constexpr (!kFull) if ((gmode & 2) && a.guideRec) {
            // A record taken at this path's previous vertex: its radiance snapshot is the sum so far
            // (that vertex's NEE included, nothing from here on), so the final sum minus it is the
            // light that came along the sampled direction.
            if (gcount > 0) {
                float4 *rec = a.guideRec + 4 * (size_t(j) * kGuideVertices + gcount - 1);
                float4 r3 = rec[3];
                if (__float_as_int(r3.w) == 1) {
                    float4 r2 = rec[2];
                    r2.w = 0.25f * (L.v[0] + L.v[1] + L.v[2] + L.v[3]);
                    rec[2] = r2;
                    rec[3] = make_float4(r3.x, r3.y, r3.z, __int_as_float(2));
                }
            }
        }

        auto misScale = [&]() {
            float av = 0.25f * (rpath.v[0] + rpath.v[1] + rpath.v[2] + rpath.v[3]);
            return av > 0.f && isfinite(av) ? 1.f / av : 0.f;
        };
        auto add = [&](SS c) {
            Lhero = Lhero + c;
            L = L + c * misScale();
        };
        // NEE: queue a shadow ray carrying f * Le * w / pdf; the visibility test adds it later.
        // The shadow ray starts in the medium on the light's side of the vertex (medIn / medOut
        // for surfaces, the current medium for medium vertices where ng = 0).
        auto nee = [&](V3 p, V3 ng, const Lobe *lobe, const Frame *fr, V3 ns, V3 wo, float g, int medIn, int medOut,
                       const GuideMix *gmix, const FullBsdf *full = nullptr) {
            float ul = rng.uniform(), u0 = rng.uniform(), u1 = rng.uniform();
            LightSample ls;
            bool picked = false;
            if constexpr (kDelta) {
                // The spot / distant / goniometric lights take the first band of ul; the light
                // sampler gets the rest, its own bands (infinite lights, then bounded lights)
                // summing to what is left.
                float acc = 0.f;
                for (int k = 0; k < s.deltaCount && !picked; ++k) {
                    const DevDelta &l = s.deltas[k];
                    if (ul < acc + l.pmf) {
                        ls = sample_delta_light(s, l, p, lam);
                        picked = true;
                    }
                    acc += l.pmf;
                }
                ul -= acc;
            }
            if (!picked) ls = sample_light(s, p, ng, lam, ul, u0, u1);
            if (!ls.ok) return;
            int med = dot(ls.wi, ng) > 0.f ? medOut : medIn;
            SS f;
            float spdf;
            if (lobe) {
                V3 wol = fr->to_local(wo), wil = fr->to_local(ls.wi);
                if (wol.z == 0.f) return;
                f = lobe_f(*lobe, wol, wil) * fabsf(dot(ls.wi, ns));
                spdf = lobe_pdf(*lobe, wol, wil);
                // Guided vertices sample from the one-sample mixture: MIS against its pdf.
                if constexpr (kGuide)
                    if (gmix)
                        spdf = gmix->c * guide_pdf_folded(*gmix, ls.wi, ns, dot(wo, ns) > 0.f ? 1.f : -1.f) +
                               (1.f - gmix->c) * spdf;
            } else if (full) {
                V3 wol = fr->to_local(wo), wil = fr->to_local(ls.wi);
                if (wol.z == 0.f) return;
                f = full_f(*full, wol, wil) * fabsf(dot(ls.wi, ns));
                spdf = full_pdf(*full, wol, wil);
            } else {
                float ph = hg_phase(dot(wo, ls.wi), g);
                f = splat(ph);
                spdf = ph;
            }
            if (!nonzero(f)) return;
            float w = ls.delta ? 1.f : power_heuristic(ls.pdf, spdf);
            SS c = beta * f * ls.Le * (w / ls.pdf);
            if (!nonzero(c)) return;
            V3 so = p + (dot(ls.target - p, ng) < 0.f ? -ng : ng) * ray_eps(p);
            int k = warp_append(a.counters + kCntShadow);
            a.S.o[k] = make_float4(so.x, so.y, so.z, __int_as_float(med));
            V3 sd = ls.target - so;
            a.S.d[k] = make_float4(sd.x, sd.y, sd.z, __int_as_float(j));
            a.S.c[k] = to_f4(c);
            a.S.w[k] = misScale();
        };
        auto roulette = [&]() {
            if (depth <= 1) return true;
            float ms = lam.terminated() ? 1.f : misScale();
            float mx = max_c(beta) * etaScale * ms;
            if (mx >= 1.f) return true;
            float qq = fmaxf(0.f, 1.f - mx);
            if (rng.uniform() < qq) return false;
            beta = beta * (1.f / (1.f - qq));
            return true;
        };

        if (iters > 8192) {
            alive = false;
            atomicOr(a.counters + kCntStatus, kStatusGuard);
        }
        bool handled = !alive;
        bool found = prim >= 0;
        // Participating medium along the segment: hero-driven free flight in homogeneous media
        // (medium.cpp:71-103, with the rPath pdf ratios of path-level spectral MIS), spectral
        // tracking in grid media (medium.cpp:232-285, wavelength-neutral: rPath unchanged).
        // The guided class holds surface hits outside media on diffuse materials only (k_classify),
        // so its launch (kGuide) compiles neither the medium, the escape nor the non-diffuse code.
        if (!kFull && !kGuide && !handled && medium >= 0) {
            float tMax = found ? hit.x : kInf;
            int event = 0;  // 0: the segment is crossed, 1: real scattering at t, 2: the path ends
            float t = tMax, g = 0.f;
            if (!is_grid(s, medium)) {
                const prgpu::Medium &md = s.media[medium];
                g = md.g;
                SS ss = tab4(s.spectra, md.sigmaS, lam) * md.scale;
                SS st = tab4(s.spectra, md.sigmaA, lam) * md.scale + ss;
                float u = fminf(rng.uniform(), kOneMinusEps);
                t = st.v[0] > 0.f ? -logf(1.f - u) / st.v[0] : kInf;
                if (t < tMax) {
                    SS T;
#pragma unroll
                    for (int i = 0; i < 4; ++i) T.v[i] = expf(-st.v[i] * t);
                    float pdf0 = st.v[0] * T.v[0];
                    if (!(pdf0 > 0.f)) {
                        event = 2;
                    } else {
                        beta = beta * T * ss * (1.f / pdf0);
                        rpath = rpath * st * T * (1.f / pdf0);
                        event = 1;
                    }
                } else {
                    SS T;
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        T.v[i] = isinf(tMax) ? (st.v[i] > 0.f ? 0.f : 1.f) : expf(-st.v[i] * tMax);
                    if (!(T.v[0] > 0.f)) {
                        event = 2;
                    } else {
                        beta = beta * T * (1.f / T.v[0]);
                        rpath = rpath * T * (1.f / T.v[0]);
                        if (!nonzero(beta)) event = 2;
                    }
                }
            } else {
                const DevGrid &gr = s.grids[medium - s.mediumCount];
                g = gr.g;
                SS wgt;
                event = grid_sample(s, gr, lam, o, d, tMax, rng, &t, &wgt);
                beta = beta * wgt;
                if (event == 0 && !nonzero(beta)) event = 2;
            }
            if (event == 2) {
                alive = false;
                handled = true;
            } else if (event == 1) {
                handled = true;
                if (!nonzero(beta) || (maxDepth > 0 && depth >= maxDepth)) {
                    alive = false;
                } else {
                    ++depth;
                    V3 p = o + d * t, wo = -d;
                    nee(p, mk(0.f, 0.f, 0.f), nullptr, nullptr, mk(0.f, 0.f, 0.f), wo, g, medium, medium, nullptr);
                    float u0 = rng.uniform(), u1 = rng.uniform(), phasePdf;
                    V3 wi = hg_sample(wo, g, u0, u1, &phasePdf);
                    if (!(phasePdf > 0.f)) {
                        alive = false;
                    } else {
                        prevPdf = phasePdf;
                        prevP = p;
                        prevN = mk(0.f, 0.f, 0.f);
                        specular = false;
                        o = p;
                        d = wi;
                        alive = roulette();
                    }
                }
            }
        }
        if (!kFull && !kGuide && !handled && !found) {
            // Escaped: emission of every infinite light with MIS against the previous BSDF /
            // phase sample.
            if (s.envSpectrum >= 0) {
                SS Le = tab4(s.spectra, s.envSpectrum, lam) * s.envScale;
                float w = 1.f;
                if (depth > 0 && !specular) w = power_heuristic(prevPdf, s.envPmf * kInv4Pi);
                add(beta * Le * w);
            }
            if (s.envMap.w > 0) {
                SS Le = env_lookup(s, d, lam);
                float w = 1.f;
                if (depth > 0 && !specular) w = power_heuristic(prevPdf, s.envMap.pmf * env_pdf(s, d));
                add(beta * Le * w);
            }
            if (s.sun.spectrum >= 0 && dot(normalize(d), s.sun.z) >= s.sun.cosMax) {
                SS Le = tab4(s.spectra, s.sun.spectrum, lam) * s.sun.scale;
                float w = 1.f;
                if (depth > 0 && !specular) w = power_heuristic(prevPdf, s.sun.pmf * sun_pdf(s.sun));
                add(beta * Le * w);
            }
            alive = false;
            handled = true;
        }
        if (!handled) {
            const prgpu::Primitive &pr = s.prims[prim];
            Surf sf = shade_point(s, pr, hit.x, hit.y, hit.z, o, d);
            if (!kFull && pr.light >= 0) {
                const prgpu::Light &l = s.lights[pr.light];
                SS Le = emitted(s, l, sf.n, -d, lam);
                if (nonzero(Le)) {
                    float w = 1.f;
                    if (depth > 0 && !specular)
                        w = power_heuristic(prevPdf, light_pmf(s, pr.light, prevP, prevN) * area_pdf(l, prevP, sf.p, sf.n));
                    add(beta * Le * w);
                }
            }
            const prgpu::Material &m = s.mats[pr.material];
            if (!kGuide && m.type == prgpu::MatInterface) {
                // Invisible medium boundary: switch media and continue straight on.
                if (++crossings > 1000) {
                    alive = false;
                } else {
                    medium = dot(d, sf.n) > 0.f ? pr.mediumOutside : pr.mediumInside;
                    o = offset_origin(sf.p, sf.n, d);
                }
            } else if ((!kGuide && m.type == prgpu::MatBlack) || (maxDepth > 0 && depth >= maxDepth)) {
                alive = false;
            } else if (!kFull && !kGuide && full_material(m)) {
                deferred = true;
            } else {
                ++depth;
                if constexpr (kDelta) perturb_shading(s, int(&m - s.mats), pr, &sf);
                Frame fr = frame_from_xz(sf.dpdu, sf.ns);
                V3 wo = -d;
                V3 wol = fr.to_local(wo);
                BSample bs;
                bool ok;
                float misPdf;  // the BSDF density for MIS against later light hits
                // Guided vertices: the sampling density over the BSDF's, folded into etaScale so
                // that Russian roulette keeps testing the throughput BSDF sampling would have given
                // (a guide that sends the path towards bright directions lowers beta there by the
                // same factor; testing beta alone would kill exactly the paths it found).
                float rrScale = 1.f;
                if constexpr (kFull) {
                    // Coats and sheen (FullBsdf: stochastic layered walks, out of line); a
                    // proportional sampling pdf takes the estimated density for MIS (path.cpp:219).
                    FullBsdf fb;
                    make_full(s, m, sf.u, sf.v, lam, &fb);
                    if constexpr (kDelta) {
                        textured_full(s, int(&m - s.mats), TexCtx{sf.p, sf.u, sf.v}, lam, &fb);
                    }
                    if (full_non_specular(fb))
                        nee(sf.p, sf.n, nullptr, &fr, sf.ns, wo, 0.f, pr.mediumInside, pr.mediumOutside, nullptr, &fb);
                    float uc = rng.uniform(), u0 = rng.uniform(), u1 = rng.uniform();
                    bool proportional = false;
                    ok = wol.z != 0.f && full_sample(fb, wol, uc, u0, u1, &bs, &proportional);
                    ok = ok && nonzero(bs.f) && bs.pdf > 0.f && isfinite(bs.pdf) && bs.wi.z != 0.f &&
                         isfinite(bs.f.v[0] + bs.f.v[1] + bs.f.v[2] + bs.f.v[3]);
                    misPdf = ok && proportional ? full_pdf(fb, wol, bs.wi) : bs.pdf;
                } else {
                Lobe lobe = kGuide ? diffuse_lobe(s, m, sf.u, sf.v, lam) : make_lobe(s, m, sf.u, sf.v, lam);
                if constexpr (kDelta) textured_lobe(s, int(&m - s.mats), TexCtx{sf.p, sf.u, sf.v}, lam, &lobe);
                if constexpr (kGuide) {
                    GuideMix gm;
                    // The guide is trained on, and applied at, the first kGuideVertices diffuse
                    // vertices of each path.
                    const bool diffuseVertex = c == kClassGuided && m.type == prgpu::MatDiffuse;
                    const bool inRange = diffuseVertex && gcount < kGuideVertices;
                    const bool guided = (gmode & 1) && inRange;
                    const int recIndex = gcount;
                    if (inRange) ++gcount;
                    if (guided) gm = guide_decode(a.guideOut + size_t(q - first) * kGuideOut, a.guideOpts);
                    if (lobe.non_specular())
                        nee(sf.p, sf.n, &lobe, &fr, sf.ns, wo, 0.f, pr.mediumInside, pr.mediumOutside,
                            guided ? &gm : nullptr);
                    float pbGuide = 0.f;
                    if (guided) {
                        // One-sample MIS of the guide and the BSDF: wi ~ c q + (1 - c) p_bsdf.
                        float us = rng.uniform(), uc = rng.uniform(), u0 = rng.uniform(), u1 = rng.uniform();
                        V3 wiw;
                        ok = wol.z != 0.f;
                        const float side = dot(wo, sf.ns) > 0.f ? 1.f : -1.f;
                        if (us < gm.c) {
                            wiw = guide_sample(gm, uc, u0, u1);
                            if (dot(wiw, sf.ns) * side < 0.f) wiw = guide_mirror(wiw, sf.ns);
                        } else {
                            BSample b2;
                            ok = ok && lobe_sample(lobe, wol, uc, u0, u1, &b2);
                            wiw = fr.from_local(b2.wi);
                        }
                        V3 wil = fr.to_local(wiw);
                        pbGuide = lobe_pdf(lobe, wol, wil);
                        bs.f = lobe_f(lobe, wol, wil);
                        bs.pdf = gm.c * guide_pdf_folded(gm, wiw, sf.ns, side) + (1.f - gm.c) * pbGuide;
                        if (pbGuide > 0.f) rrScale = fminf(fmaxf(bs.pdf / pbGuide, 1e-3f), 1e3f);
                        bs.wi = wil;
                        bs.flags = kFlagReflection | kFlagDiffuse;
                        bs.eta = 1.f;
                    } else {
                        float uc = rng.uniform(), u0 = rng.uniform(), u1 = rng.uniform();
                        ok = wol.z != 0.f && lobe.flags() != 0u && lobe_sample(lobe, wol, uc, u0, u1, &bs);
                    }
                    ok = ok && nonzero(bs.f) && bs.pdf > 0.f && isfinite(bs.pdf) && bs.wi.z != 0.f &&
                         isfinite(bs.f.v[0] + bs.f.v[1] + bs.f.v[2] + bs.f.v[3]);
                    float4 *rec = a.guideRec + 4 * (size_t(j) * kGuideVertices + recIndex);
                    if (ok && (gmode & 2) && inRange) {
                        // First diffuse vertex of the path: record (x, n, wo, wi, p_bsdf, mean beta).
                        const float *bmin = s.root.box, *bmax = s.root.box + 3;
                        V3 xn = mk((sf.p.x - bmin[0]) / fmaxf(bmax[0] - bmin[0], 1e-20f),
                                   (sf.p.y - bmin[1]) / fmaxf(bmax[1] - bmin[1], 1e-20f),
                                   (sf.p.z - bmin[2]) / fmaxf(bmax[2] - bmin[2], 1e-20f));
                        V3 wiw = fr.from_local(bs.wi);
                        float pbr = guided ? pbGuide : lobe_pdf(lobe, wol, bs.wi);
                        float bavg = 0.25f * (beta.v[0] + beta.v[1] + beta.v[2] + beta.v[3]);
                        rec[0] = make_float4(xn.x, xn.y, xn.z, bavg);
                        rec[1] = make_float4(sf.ns.x, sf.ns.y, sf.ns.z, pbr);
                        rec[2] = make_float4(wo.x, wo.y, wo.z, 0.f);
                        rec[3] = make_float4(wiw.x, wiw.y, wiw.z, __int_as_float(1));
                    }
                } else {
                    if (lobe.non_specular())
                        nee(sf.p, sf.n, &lobe, &fr, sf.ns, wo, 0.f, pr.mediumInside, pr.mediumOutside, nullptr);
                    float uc = rng.uniform(), u0 = rng.uniform(), u1 = rng.uniform();
                    ok = wol.z != 0.f && lobe.flags() != 0u && lobe_sample(lobe, wol, uc, u0, u1, &bs);
                    ok = ok && nonzero(bs.f) && bs.pdf > 0.f && isfinite(bs.pdf) && bs.wi.z != 0.f &&
                         isfinite(bs.f.v[0] + bs.f.v[1] + bs.f.v[2] + bs.f.v[3]);
                }
                misPdf = bs.pdf;
                }
                if (!ok) {
                    alive = false;
                } else {
                    V3 wi = fr.from_local(bs.wi);
                    beta = beta * bs.f * (fabsf(dot(wi, sf.ns)) / bs.pdf);
                    prevPdf = misPdf;
                    specular = (bs.flags & kFlagSpecular) != 0u;
                    if (bs.flags & kFlagTransmission) etaScale *= sqr(bs.eta);
                    etaScale *= rrScale;
                    prevP = sf.p;
                    prevN = sf.n;
                    o = offset_origin(sf.p, sf.n, wi);
                    d = wi;
                    // Medium on the side the new direction enters.
                    medium = dot(wi, sf.n) > 0.f ? pr.mediumOutside : pr.mediumInside;
                    if (!nonzero(beta) || !isfinite(max_c(beta))) alive = false;
                    else alive = roulette();
                }
            }
        }
        // Write back (the radiance sums always; the ray state only for survivors).
        P.L[j] = to_f4(L);
        P.Lhero[j] = to_f4(Lhero);
        P.lpdf[j] = make_float4(lam.pdf[0], lam.pdf[1], lam.pdf[2], lam.pdf[3]);
        if (alive) {
            P.o[j] = make_float4(o.x, o.y, o.z, prevPdf);
            P.d[j] = make_float4(d.x, d.y, d.z, etaScale);
            P.beta[j] = to_f4(beta);
            P.rpath[j] = to_f4(rpath);
            P.rng[j] = make_ulonglong2(rng.state, rng.inc);
            P.meta[j] = make_int4(meta.x, depth, medium,
                                  (specular ? 1 : 0) | (gcount << 2) | (min(crossings, 0xffff) << 8) |
                                      (flags & (0xff << kRenderShift)));
            P.prevP[j] = make_float4(prevP.x, prevP.y, prevP.z, pp4.w);
            P.prevN[j] = make_float4(prevN.x, prevN.y, prevN.z, __int_as_float(iters));
            if (!kFull && deferred) {
                a.fullQ[warp_append(a.counters + kCntFull)] = j;
                continue;
            }
            a.queueOut[warp_append(a.counters + kCntNext)] = j;
            if (kBatch) {
                // Survivors per slot half (warp-aggregated): the batch loop films a wave once its
                // half has none left.
                unsigned m = __activemask(), m1 = __ballot_sync(m, j >= a.halfSlots);
                if ((threadIdx.x & 31) == __ffs(m) - 1) {
                    if (m1) atomicAdd(a.counters + kCntNextLive1, __popc(m1));
                    if (m & ~m1) atomicAdd(a.counters + kCntNextLive0, __popc(m & ~m1));
                }
            }
        }
    }
}

// An unoccluded NEE sample: its contribution times the transmittance of the medium it crossed
// goes to the path's radiance sums (one shadow entry per path and bounce, so no atomics).
template <bool kMedia>
__device__ __forceinline__ void shadow_accept(const DevScene &s, const Paths &P, const Shadows &S, int q) {
    float4 o4 = S.o[q], d4 = S.d[q];
    int medium = __float_as_int(o4.w), j = __float_as_int(d4.w);
    SS c = from_f4(S.c[q]);
    if (kMedia && medium >= 0) c = c * segment_tr(s, medium, load_lam(P, j), mk(o4.x, o4.y, o4.z), mk(d4.x, d4.y, d4.z), 1.f);
    float w = S.w[q];
    float4 L = P.L[j], Lh = P.Lhero[j];
    P.L[j] = make_float4(L.x + c.v[0] * w, L.y + c.v[1] * w, L.z + c.v[2] * w, L.w + c.v[3] * w);
    P.Lhero[j] = make_float4(Lh.x + c.v[0], Lh.y + c.v[1], Lh.z + c.v[2], Lh.w + c.v[3]);
}

// Visibility of queued NEE samples: any-hit queries up to 1 - ShadowEpsilon of the segment, by
// persistent warps with lane refill. kMedia: the scene has media, so accepted segments carry a
// transmittance (kept out of the medium-free variant, whose traversal loop would otherwise pay
// registers for the ratio-tracking code). kWalls: the scene has medium interfaces; they are
// transparent to this query, an occluded segment is done, an unoccluded one that crossed no
// interface stays in its starting medium, and the rest go to the walk queue (k_shadow_walk).
template <bool kSpheres, bool kMedia, bool kBatch = false, bool kWalls = false>
__global__ void __launch_bounds__(256, (kSpheres || kMedia || kWalls) ? 1 : 4)
    k_shadow_any(DevScene s0, const DevScene *scenes, Paths P, Shadows S, int *counters) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int n = counters[kCntShadow];
    __shared__ int2 shortStack[kShortStack * 256];
    HybridStack<kShortStack, 256> hs;
    hs.sh = shortStack + threadIdx.x;
    TraceRay r;
    TravState st;
    st.ref = 0;
    st.sp = 0;
    st.tMax = 1.f - kShadowEps;
    st.found = false;
    st.crossed = false;
    int q = 0, rid = 0;
    const QNode *nodes = s0.qnodes;
    const LeafPrim *leaves = s0.leaves;
    const uint8_t *cls = s0.primClass;
    // pending: this lane's segment is traced and its outcome (accept, walk or occluded) not yet
    // applied; that happens when the lane takes its next entry (kRefillLanes).
    bool active = false, exhausted = n == 0, pending = false, overflow = false;
    while (!__all_sync(full, exhausted)) {
        const bool idle = !active && !exhausted;
        const unsigned need = __ballot_sync(full, idle), busy = __ballot_sync(full, active);
        if (need && (__popc(need) >= kRefillLanes || !busy)) {
            bool toWalk = false;
            if (idle && pending && !st.found) {
                if (kWalls && st.crossed) toWalk = true;
                else shadow_accept<kMedia>(SceneOf<kBatch>::get(s0, scenes, rid), P, S, q);
            }
            pending = false;
            if (kWalls) {
                const unsigned m = __ballot_sync(full, toWalk);
                if (m) {
                    const int leader = __ffs(m) - 1;
                    int wb = 0;
                    if (lane == leader) wb = atomicAdd(counters + kCntWalk, __popc(m));
                    wb = __shfl_sync(full, wb, leader);
                    if (toWalk) S.walk[wb + __popc(m & ((1u << lane) - 1u))] = q;
                }
            }
            int base = 0;
            if (lane == 0) base = atomicAdd(counters + kCntShadowWork, __popc(need));
            base = __shfl_sync(full, base, 0);
            if (idle) {
                q = base + __popc(need & ((1u << lane) - 1u));
                if (q >= n) {
                    exhausted = true;
                } else {
                    float4 o4 = S.o[q], d4 = S.d[q];
                    if (kBatch) rid = path_render(P.meta[__float_as_int(d4.w)].w);
                    const DevScene &s = SceneOf<kBatch>::get(s0, scenes, rid);
                    nodes = s.qnodes;
                    leaves = s.leaves;
                    cls = s.primClass;
                    r = make_trace_ray(mk(o4.x, o4.y, o4.z), mk(d4.x, d4.y, d4.z));
                    st.tMax = 1.f - kShadowEps;
                    st.sp = 0;
                    st.found = false;
                    st.crossed = false;
                    float te;
                    active = !s.root.empty &&
                             box_entry(r, s.root.box[0], s.root.box[1], s.root.box[2], s.root.box[3], s.root.box[4],
                                       s.root.box[5], &te) &&
                             te < st.tMax;
                    st.ref = s.root.ref;
                    // A segment that misses the root box: unoccluded, accepted at the next refill.
                    pending = !active;
                }
            }
        }
        if (active && traverse4_step_st<true, kSpheres, kWalls>(nodes, leaves, r, st, hs, &overflow, cls)) {
            active = false;
            pending = true;
        }
    }
    if (overflow) atomicOr(counters + kCntStatus, kStatusStack);
}

// Moves the survivors' queue into place for the next bounce and accumulates statistics (one
// thread; keeps the bounce loop free of host round trips).
static __global__ void k_advance(int *counters, unsigned long long *stats) {
    stats[kStatClosest] += (unsigned long long)counters[kCntActive];
    stats[kStatShadow] += (unsigned long long)counters[kCntShadow];
    stats[kStatBounces] += counters[kCntActive] > 0 ? 1ull : 0ull;
    counters[kCntActive] = counters[kCntNext];
    counters[kCntNext] = 0;
    counters[kCntLive0] = counters[kCntNextLive0];
    counters[kCntLive1] = counters[kCntNextLive1];
    counters[kCntNextLive0] = 0;
    counters[kCntNextLive1] = 0;
    counters[kCntShadow] = 0;
    counters[kCntExtendWork] = 0;
    counters[kCntShadowWork] = 0;
    counters[kCntWalk] = 0;
    counters[kCntFull] = 0;
#pragma unroll
    for (int c = 0; c < kClasses; ++c) counters[kCntClass0 + c] = 0;
}

// Closest hit of a ray on the 4-wide tree within [0, tMax) (one thread, whole traversal).
template <bool kSpheres>
__device__ __forceinline__ bool closest4(const DevScene &s, const TraceRay &r, float tMax, Hit *h, bool *overflow) {
    float te;
    if (s.root.empty ||
        !box_entry(r, s.root.box[0], s.root.box[1], s.root.box[2], s.root.box[3], s.root.box[4], s.root.box[5], &te) ||
        !(te < tMax))
        return false;
    int stackRef[kStackSize];
    float stackT[kStackSize];
    TravState st;
    st.ref = s.root.ref;
    st.sp = 0;
    st.tMax = tMax;
    st.found = false;
    st.crossed = false;
    while (!traverse4_step<false, kSpheres>(s.qnodes, s.leaves, r, st, stackRef, stackT, overflow)) {
    }
    if (st.found) *h = st.hit;
    return st.found;
}

// Closest medium interface along a ray within [0, tMax): brute force over the scene's short
// interface list (the leaf slots' own hit arithmetic), else the whole tree.
template <bool kSpheres>
__device__ __forceinline__ bool closest_wall(const DevScene &s, const TraceRay &r, float tMax, Hit *h, bool *overflow) {
    if (s.wallCount < 0) return closest4<kSpheres>(s, r, tMax, h, overflow);
    bool found = false;
    for (int i = 0; i < s.wallCount; ++i) {
        const LeafPrim *p = s.walls + i;
        float4 v0 = __ldg(&p->v0), v1 = __ldg(&p->v1), v2 = __ldg(&p->v2);
        float t, u = 0.f, v = 0.f;
        bool hh;
        if (kSpheres && __float_as_int(v1.w) == 1)
            hh = hit_sphere(r, v0, v1, tMax, &t);
        else
            hh = hit_triangle(r, v0, v1, v2, tMax, &t, &u, &v);
        if (hh) {
            tMax = t;
            h->t = t;
            h->u = u;
            h->v = v;
            h->prim = __float_as_int(v0.w);
            found = true;
        }
    }
    return found;
}

// The queued NEE samples whose segment crosses a medium interface: a walk through the boundary
// surfaces with each medium's transmittance (src/scene/scene.cpp:41-59). k_shadow_any has
// already found these segments free of opaque surfaces, so each step needs only the nearest
// interface.
template <bool kSpheres, bool kBatch = false>
__global__ void __launch_bounds__(256) k_shadow_walk(DevScene s0, const DevScene *scenes, Paths P, Shadows S,
                                                     int *counters) {
    int n = counters[kCntWalk];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int q = S.walk[i];
        float4 o4 = S.o[q], d4 = S.d[q];
        int medium = __float_as_int(o4.w), j = __float_as_int(d4.w);
        const DevScene &s = SceneOf<kBatch>::get(s0, scenes, path_render(P.meta[j].w));
        V3 o = mk(o4.x, o4.y, o4.z), dd = mk(d4.x, d4.y, d4.z);
        V3 target = o + dd;
        SS T = splat(1.f);
        bool overflow = false;
        Lambda lam = load_lam(P, j);
        bool blocked = true;
        for (int it = 0; it < 256; ++it) {
            V3 d = target - o;
            TraceRay r = make_trace_ray(o, d);
            Hit h;
            h.prim = -1;
            bool hit = closest_wall<kSpheres>(s, r, 1.f - kShadowEps, &h, &overflow);
            if (hit && !(__ldg(s.primClass + h.prim) & kTransparentBit)) break;
            if (medium >= 0) T = T * segment_tr(s, medium, lam, o, d, hit ? h.t : 1.f);
            if (!hit || !nonzero(T)) {
                blocked = false;
                break;
            }
            const prgpu::Primitive &pr = s.prims[h.prim];
            Surf sf = shade_point(s, pr, h.t, h.u, h.v, o, d);
            medium = dot(d, sf.n) > 0.f ? pr.mediumOutside : pr.mediumInside;
            o = offset_origin(sf.p, sf.n, d);
        }
        if (overflow) atomicOr(counters + kCntStatus, kStatusStack);
        if (blocked) continue;
        SS c = from_f4(S.c[q]) * T;
        float w = S.w[q];
        float4 L = P.L[j], Lh = P.Lhero[j];
        P.L[j] = make_float4(L.x + c.v[0] * w, L.y + c.v[1] * w, L.z + c.v[2] * w, L.w + c.v[3] * w);
        P.Lhero[j] = make_float4(Lh.x + c.v[0], Lh.y + c.v[1], Lh.z + c.v[2], Lh.w + c.v[3]);
    }
}

// Adds each sample's XYZ to the FP64 film, one sample at a time in sample-index order
// (src/gpu/prender_gpu.cpp:1541-1559 for the per-sample conversion and clamp).
// Pixel pl of a chunk whose sample k sits in path slot base + k * npix: its samples' XYZ added to
// film3 (X, Y, Z of that pixel) in sample order.
__device__ __forceinline__ void film_pixel(const DevScene &s, const Paths &P, int base, int npix, int pl, int samples,
                                           float clampY, double *film3) {
    double X = film3[0], Y = film3[1], Z = film3[2];
    for (int sIdx = 0; sIdx < samples; ++sIdx) {
        int j = base + sIdx * npix + pl;
        float fw = P.prevP[j].w;
        if (fw == 0.f) continue;
        Lambda lam = load_lam(P, j);
        SS L = from_f4(lam.terminated() ? P.Lhero[j] : P.L[j]);
        if (!isfinite(L.v[0] + L.v[1] + L.v[2] + L.v[3])) continue;
        float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (lam.pdf[i] == 0.f) continue;
            float v = L.v[i] / lam.pdf[i];
            sx += cie_x(lam.l[i]) * v;
            sy += cie_y(lam.l[i]) * v;
            sz += cie_z(lam.l[i]) * v;
        }
        float k = fw;
        if (clampY > 0.f && sy * s.norm > clampY) k *= clampY / (sy * s.norm);
        k *= s.norm;
        X += double(sx * k);
        Y += double(sy * k);
        Z += double(sz * k);
    }
    film3[0] = X;
    film3[1] = Y;
    film3[2] = Z;
}

static __global__ void __launch_bounds__(256) k_film(DevScene s, Paths P, ChunkInfo ci, float clampY, double *film) {
    for (int pl = blockIdx.x * blockDim.x + threadIdx.x; pl < ci.npix; pl += gridDim.x * blockDim.x)
        film_pixel(s, P, 0, ci.npix, pl, ci.samples, clampY, film + 3 * size_t(ci.pixBegin + pl));
}

} // namespace prb
