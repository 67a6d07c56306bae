// Coated materials and sheen on the device: the reference's LayeredBxDF (a dielectric coat over a
// diffuse or conductor base with an optional scattering layer between them, two-sided,
// src/materials/bxdf.cpp:260-518, the layered BxDF of pbrt-v4) and SheenBxDF (the "Charlie"
// sheen lobe of Estevez and Kulla over any base, bxdf.cpp:520-631). The layered f, pdf and sample
// are stochastic random walks between the two interfaces; their random numbers come from a PCG
// stream seeded by the directions (and the sample's own uniforms), so every evaluation is a
// deterministic, unbiased estimate. They stay out of line: inlined into the shading kernel they
// would cost every material registers.
#pragma once

#include "bsdf.cuh"

namespace prb {

constexpr int kSheenMuBins = 32, kSheenAlphaBins = 16;  // sheen albedo table: [alpha][mu]

struct Layered {
    Lobe top, bottom;  // dielectric coat; diffuse or conductor base
    float thickness, g;
    SS albedo;  // single-scattering albedo of the layer between the interfaces
    bool hasAlbedo;
    int maxDepth, nSamples;
};

struct Sheen {
    SS color;
    float alpha, weight, colorMax;
    const float *table;  // kSheenAlphaBins x kSheenMuBins directional albedo
};

// A surface BSDF of the coated / sheen kind: one lobe or a layered coat, optionally under sheen.
struct FullBsdf {
    Lobe base;  // the single lobe when !layered
    Layered lay;
    Sheen sh;
    bool layered, sheen, black;
};

__device__ __forceinline__ float layer_tr(float dz, V3 w) {
    if (fabsf(dz) <= 1.17549435e-38f) return 1.f;
    return expf(-fabsf(dz / w.z));
}

__device__ __forceinline__ bool good(bool ok, const BSample &s) { return ok && nonzero(s.f) && s.pdf > 0.f && s.wi.z != 0.f; }

__device__ __forceinline__ uint64_t dir_hash(V3 a, uint64_t h) {
    h = mix_bits(h ^ __float_as_uint(a.x));
    h = mix_bits(h ^ (uint64_t(__float_as_uint(a.y)) << 20));
    return mix_bits(h ^ (uint64_t(__float_as_uint(a.z)) << 40));
}

__device__ __forceinline__ Pcg walk_stream(V3 a, uint64_t sa, V3 b, uint64_t sb) {
    Pcg r;
    r.seed(dir_hash(a, sa), dir_hash(b, sb));
    return r;
}

__device__ __forceinline__ bool layered_non_specular(const Layered &l) {
    return !l.top.specular() || !l.bottom.specular() || l.hasAlbedo;
}

// Stochastic estimate of the layered BSDF value (LayeredBxDF::f, bxdf.cpp:270-376).
static __device__ __noinline__ SS layered_f(const Layered &b, V3 wo, V3 wi, bool radiance) {
    SS f = splat(0.f);
    if (wo.z < 0.f) {  // two-sided: the walk always enters through the coat
        wo = -wo;
        wi = -wi;
    }
    const bool same = same_hemi(wo, wi);
    // Leaving on wo's side means leaving through the coat; the other side, through the base.
    const Lobe &exitI = same ? b.top : b.bottom;
    const Lobe &nonExit = same ? b.bottom : b.top;
    const float exitZ = same ? b.thickness : 0.f;
    const bool exitSpec = exitI.specular(), nonExitSpec = nonExit.specular();
    if (same) f = lobe_f(b.top, wo, wi, radiance) * float(b.nSamples);
    Pcg r = walk_stream(wo, 0x3c1, wi, 0x5e7);
    for (int s = 0; s < b.nSamples; ++s) {
        BSample wos, wis;
        float u0 = r.uniform(), u1 = r.uniform(), u2 = r.uniform();
        if (!good(lobe_sample(b.top, wo, u0, u1, u2, &wos, radiance, kSampleT), wos)) continue;
        u0 = r.uniform(), u1 = r.uniform(), u2 = r.uniform();
        if (!good(lobe_sample(exitI, wi, u0, u1, u2, &wis, !radiance, kSampleT), wis)) continue;
        SS beta = wos.f * (fabsf(wos.wi.z) / wos.pdf);
        float z = b.thickness;
        V3 w = wos.wi;
        for (int depth = 0; depth < b.maxDepth; ++depth) {
            if (depth > 3 && max_c(beta) < 0.25f) {
                float q = fmaxf(0.f, 1.f - max_c(beta));
                if (r.uniform() < q) break;
                beta = beta * (1.f / (1.f - q));
            }
            if (!b.hasAlbedo) {
                z = (z == b.thickness) ? 0.f : b.thickness;
                beta = beta * layer_tr(b.thickness, w);
            } else {
                float dz = -logf(1.f - r.uniform()) * fabsf(w.z);
                float zp = w.z > 0.f ? z + dz : z - dz;
                if (0.f < zp && zp < b.thickness) {
                    // Scattering inside the layer: NEE through the exit interface, then the phase
                    // function continues the walk.
                    float wt = 1.f;
                    float phaseExit = hg_phase(dot(-w, -wis.wi), b.g);
                    if (!exitSpec) wt = power_heuristic(wis.pdf, phaseExit);
                    f = f + beta * b.albedo * wis.f * (phaseExit * wt * layer_tr(zp - exitZ, wis.wi) / wis.pdf);
                    float p0 = r.uniform(), p1 = r.uniform(), phasePdf;
                    V3 wp = hg_sample(-w, b.g, p0, p1, &phasePdf);
                    if (phasePdf == 0.f || wp.z == 0.f) continue;
                    beta = beta * b.albedo;
                    w = wp;
                    z = zp;
                    if (((z < exitZ && w.z > 0.f) || (z > exitZ && w.z < 0.f)) && !exitSpec) {
                        SS fExit = lobe_f(exitI, -w, wi, radiance);
                        if (nonzero(fExit)) {
                            float exitPdf = lobe_pdf(exitI, -w, wi, kSampleT);
                            f = f + beta * fExit * (layer_tr(zp - exitZ, wp) * power_heuristic(phasePdf, exitPdf));
                        }
                    }
                    continue;
                }
                z = clampf(zp, 0.f, b.thickness);
            }
            BSample bs;
            if (z == exitZ) {
                float e0 = r.uniform(), e1 = r.uniform(), e2 = r.uniform();
                if (!good(lobe_sample(exitI, -w, e0, e1, e2, &bs, radiance, kSampleR), bs)) break;
                beta = beta * bs.f * (fabsf(bs.wi.z) / bs.pdf);
                w = bs.wi;
            } else {
                if (!nonExitSpec) {
                    float wt = 1.f;
                    if (!exitSpec) wt = power_heuristic(wis.pdf, lobe_pdf(nonExit, -w, -wis.wi));
                    f = f + beta * lobe_f(nonExit, -w, -wis.wi, radiance) * wis.f *
                                (fabsf(wis.wi.z) * wt * layer_tr(b.thickness, wis.wi) / wis.pdf);
                }
                float e0 = r.uniform(), e1 = r.uniform(), e2 = r.uniform();
                if (!good(lobe_sample(nonExit, -w, e0, e1, e2, &bs, radiance, kSampleR), bs)) break;
                beta = beta * bs.f * (fabsf(bs.wi.z) / bs.pdf);
                w = bs.wi;
                if (!exitSpec) {
                    SS fExit = lobe_f(exitI, -w, wi, radiance);
                    if (nonzero(fExit)) {
                        float wt = 1.f;
                        if (!nonExitSpec) wt = power_heuristic(bs.pdf, lobe_pdf(exitI, -w, wi, kSampleT));
                        f = f + beta * fExit * (layer_tr(b.thickness, bs.wi) * wt);
                    }
                }
            }
        }
    }
    return f * (1.f / float(b.nSamples));
}

// Layered sampling (LayeredBxDF::Sample_f, bxdf.cpp:378-455): a coat reflection is returned as
// it is; otherwise the walk runs until it leaves through an interface. Both results carry a pdf
// that is only proportional (*proportional = true): the path tracer takes layered_pdf for MIS.
static __device__ __noinline__ bool layered_sample(const Layered &b, V3 wo, float uc, float u0, float u1, bool radiance,
                                            BSample *out) {
    bool flip = false;
    if (wo.z < 0.f) {
        wo = -wo;
        flip = true;
    }
    BSample bs;
    if (!good(lobe_sample(b.top, wo, uc, u0, u1, &bs, radiance), bs)) return false;
    if (bs.flags & kFlagReflection) {
        if (flip) bs.wi = -bs.wi;
        *out = bs;
        return true;
    }
    V3 w = bs.wi;
    bool specularPath = (bs.flags & kFlagSpecular) != 0u;
    Pcg r = walk_stream(wo, 0x1d3, mk(uc, u0, u1), 0x6b5);
    SS f = bs.f * fabsf(bs.wi.z);
    float pdf = bs.pdf;
    float z = b.thickness;
    for (int depth = 0; depth < b.maxDepth; ++depth) {
        float rrBeta = max_c(f) / pdf;
        if (depth > 3 && rrBeta < 0.25f) {
            float q = fmaxf(0.f, 1.f - rrBeta);
            if (r.uniform() < q) return false;
            pdf *= 1.f - q;
        }
        if (w.z == 0.f) return false;
        if (b.hasAlbedo) {
            float dz = -logf(1.f - r.uniform()) * fabsf(w.z);
            float zp = w.z > 0.f ? z + dz : z - dz;
            if (zp == z) return false;
            if (0.f < zp && zp < b.thickness) {
                float p0 = r.uniform(), p1 = r.uniform(), phasePdf;
                V3 wp = hg_sample(-w, b.g, p0, p1, &phasePdf);
                if (phasePdf == 0.f || wp.z == 0.f) return false;
                f = f * b.albedo * phasePdf;
                pdf *= phasePdf;
                specularPath = false;
                w = wp;
                z = zp;
                continue;
            }
            z = clampf(zp, 0.f, b.thickness);
        } else {
            z = (z == b.thickness) ? 0.f : b.thickness;
            f = f * layer_tr(b.thickness, w);
        }
        const Lobe &iface = (z == 0.f) ? b.bottom : b.top;
        float e0 = r.uniform(), e1 = r.uniform(), e2 = r.uniform();
        BSample s2;
        if (!good(lobe_sample(iface, -w, e0, e1, e2, &s2, radiance), s2)) return false;
        f = f * s2.f;
        pdf *= s2.pdf;
        specularPath = specularPath && (s2.flags & kFlagSpecular);
        w = s2.wi;
        if (s2.flags & kFlagTransmission) {
            uint32_t flags = same_hemi(wo, w) ? kFlagReflection : kFlagTransmission;
            flags |= specularPath ? kFlagSpecular : kFlagGlossy;
            if (flip) w = -w;
            out->f = f;
            out->wi = w;
            out->pdf = pdf;
            out->flags = flags;
            out->eta = 1.f;
            return true;
        }
        f = f * fabsf(s2.wi.z);
    }
    return false;
}

// Stochastic estimate of the layered pdf (LayeredBxDF::PDF, bxdf.cpp:457-518), mixed with a
// uniform sphere density (weight 0.1) as the reference does.
static __device__ __noinline__ float layered_pdf(const Layered &b, V3 wo, V3 wi, bool radiance) {
    if (wo.z < 0.f) {
        wo = -wo;
        wi = -wi;
    }
    Pcg r = walk_stream(wi, 0x2a9, wo, 0x71f);
    const bool same = same_hemi(wo, wi);
    float pdfSum = same ? float(b.nSamples) * lobe_pdf(b.top, wo, wi, kSampleR) : 0.f;
    for (int s = 0; s < b.nSamples; ++s) {
        BSample wos, wis;
        if (same) {
            // Transmission through the coat both ways, one bounce off the base in between.
            const Lobe &tI = b.top, &rI = b.bottom;
            float a0 = r.uniform(), a1 = r.uniform(), a2 = r.uniform();
            bool okO = good(lobe_sample(tI, wo, a0, a1, a2, &wos, radiance, kSampleT), wos);
            float c0 = r.uniform(), c1 = r.uniform(), c2 = r.uniform();
            bool okI = good(lobe_sample(tI, wi, c0, c1, c2, &wis, !radiance, kSampleT), wis);
            if (!(okO && okI)) continue;
            if (tI.specular()) {
                pdfSum += lobe_pdf(rI, -wos.wi, -wis.wi);
            } else {
                float d0 = r.uniform(), d1 = r.uniform(), d2 = r.uniform();
                BSample rs;
                if (!good(lobe_sample(rI, -wos.wi, d0, d1, d2, &rs, radiance), rs)) continue;
                if (rI.specular()) {
                    pdfSum += lobe_pdf(tI, -rs.wi, wi);
                } else {
                    float rPdf = lobe_pdf(rI, -wos.wi, -wis.wi);
                    pdfSum += power_heuristic(wis.pdf, rPdf) * rPdf;
                    float tPdf = lobe_pdf(tI, -rs.wi, wi);
                    pdfSum += power_heuristic(rs.pdf, tPdf) * tPdf;
                }
            }
        } else {
            const Lobe &toI = b.top, &tiI = b.bottom;
            float a0 = r.uniform(), a1 = r.uniform(), a2 = r.uniform();
            if (!good(lobe_sample(toI, wo, a0, a1, a2, &wos, radiance), wos) || (wos.flags & kFlagReflection)) continue;
            float c0 = r.uniform(), c1 = r.uniform(), c2 = r.uniform();
            if (!good(lobe_sample(tiI, wi, c0, c1, c2, &wis, !radiance), wis) || (wis.flags & kFlagReflection)) continue;
            if (toI.specular())
                pdfSum += lobe_pdf(tiI, -wos.wi, wi);
            else if (tiI.specular())
                pdfSum += lobe_pdf(toI, wo, -wis.wi);
            else
                pdfSum += 0.5f * (lobe_pdf(toI, wo, -wis.wi) + lobe_pdf(tiI, -wos.wi, wi));
        }
    }
    return 0.1f * kInv4Pi + 0.9f * pdfSum / float(b.nSamples);
}

// ---------------------------------------------------------------------------------------------
// Sheen

__device__ __forceinline__ float sheen_albedo(const Sheen &sh, float cosTheta) {
    float fa = (clampf(sh.alpha, 0.05f, 1.f) - 0.05f) / 0.95f * float(kSheenAlphaBins - 1);
    float fm = clampf(fabsf(cosTheta), 0.f, 1.f) * float(kSheenMuBins - 1);
    int ia = min(int(fa), kSheenAlphaBins - 2), im = min(int(fm), kSheenMuBins - 2);
    float ta = fa - float(ia), tm = fm - float(im);
    const float *t0 = sh.table + ia * kSheenMuBins, *t1 = t0 + kSheenMuBins;
    float l0 = __ldg(t0 + im) + (__ldg(t0 + im + 1) - __ldg(t0 + im)) * tm;
    float l1 = __ldg(t1 + im) + (__ldg(t1 + im + 1) - __ldg(t1 + im)) * tm;
    return l0 + (l1 - l0) * ta;
}

// Charlie distribution with the visibility term 1 / (4 (cos_i + cos_o - cos_i cos_o)).
__device__ __forceinline__ float sheen_value(V3 wo, V3 wi, float alpha) {
    if (!same_hemi(wo, wi)) return 0.f;
    float co = fabsf(wo.z), ci = fabsf(wi.z);
    if (co == 0.f || ci == 0.f) return 0.f;
    V3 wh = normalize(wo + wi);
    float inv = 1.f / alpha;
    float sin2 = fmaxf(0.f, 1.f - wh.z * wh.z);
    float D = (2.f + inv) * powf(sin2, 0.5f * inv) * kInv2Pi;
    return D / (4.f * (ci + co - ci * co));
}

// ---------------------------------------------------------------------------------------------
// The composed BSDF (SheenBxDF over a lobe or a layered coat), local frame.

__device__ __forceinline__ bool full_base_non_specular(const FullBsdf &b) {
    if (b.black) return false;
    return b.layered ? layered_non_specular(b.lay) : !b.base.specular();
}
__device__ __forceinline__ bool full_non_specular(const FullBsdf &b) { return b.sheen || full_base_non_specular(b); }

__device__ __forceinline__ SS full_base_f(const FullBsdf &b, V3 wo, V3 wi) {
    if (b.black) return splat(0.f);
    return b.layered ? layered_f(b.lay, wo, wi, true) : lobe_f(b.base, wo, wi, true);
}
__device__ __forceinline__ float full_base_pdf(const FullBsdf &b, V3 wo, V3 wi) {
    if (b.black) return 0.f;
    return b.layered ? layered_pdf(b.lay, wo, wi, true) : lobe_pdf(b.base, wo, wi);
}
__device__ __forceinline__ float sheen_base_scale(const FullBsdf &b, V3 wo, V3 wi) {
    float e = fmaxf(sheen_albedo(b.sh, wo.z), sheen_albedo(b.sh, wi.z));
    return fmaxf(0.f, 1.f - b.sh.weight * b.sh.colorMax * e);
}
__device__ __forceinline__ float sheen_prob(const FullBsdf &b, V3 wo) {
    if (b.black) return 1.f;
    return clampf(b.sh.weight * b.sh.colorMax * sheen_albedo(b.sh, wo.z), 0.f, 0.9f);
}

static __device__ __noinline__ SS full_f(const FullBsdf &b, V3 wo, V3 wi) {
    if (!b.sheen) return full_base_f(b, wo, wi);
    return b.sh.color * (b.sh.weight * sheen_value(wo, wi, b.sh.alpha)) + full_base_f(b, wo, wi) * sheen_base_scale(b, wo, wi);
}

static __device__ __noinline__ float full_pdf(const FullBsdf &b, V3 wo, V3 wi) {
    if (!b.sheen) return full_base_pdf(b, wo, wi);
    float ps = sheen_prob(b, wo);
    float pdfSheen = same_hemi(wo, wi) ? fabsf(wi.z) * kInvPi : 0.f;
    return ps * pdfSheen + (1.f - ps) * full_base_pdf(b, wo, wi);
}

// Sampling (SheenBxDF::Sample_f over LayeredBxDF / a lobe). *proportional: the pdf is only
// proportional to the sampling density (the path tracer then takes full_pdf for MIS).
static __device__ __noinline__ bool full_sample(const FullBsdf &b, V3 wo, float uc, float u0, float u1, BSample *s,
                                         bool *proportional) {
    *proportional = false;
    if (!b.sheen) {
        if (b.black) return false;
        if (!b.layered) return lobe_sample(b.base, wo, uc, u0, u1, s);
        *proportional = true;
        return layered_sample(b.lay, wo, uc, u0, u1, true, s);
    }
    const float ps = sheen_prob(b, wo);
    const bool exact = !b.layered;
    if (uc < ps) {
        V3 wi = cosine_hemisphere(u0, u1);
        if (wo.z < 0.f) wi.z = -wi.z;
        s->wi = wi;
        s->flags = kFlagReflection | kFlagGlossy;
        s->eta = 1.f;
        if (exact) {
            float pdf = full_pdf(b, wo, wi);
            if (pdf == 0.f) return false;
            s->f = full_f(b, wo, wi);
            s->pdf = pdf;
        } else {
            s->f = b.sh.color * (b.sh.weight * sheen_value(wo, wi, b.sh.alpha));
            s->pdf = ps * fabsf(wi.z) * kInvPi;
            *proportional = true;
        }
        return true;
    }
    float uc2 = ps < 1.f ? fminf((uc - ps) / (1.f - ps), kOneMinusEps) : 0.f;
    bool baseProportional = false;
    bool ok = b.black ? false
                      : (b.layered ? (baseProportional = true, layered_sample(b.lay, wo, uc2, u0, u1, true, s))
                                   : lobe_sample(b.base, wo, uc2, u0, u1, s));
    if (!ok || s->pdf == 0.f) return false;
    const bool specular = (s->flags & kFlagSpecular) != 0u;
    if (specular || !exact || baseProportional) {
        s->f = s->f * sheen_base_scale(b, wo, s->wi);
        s->pdf *= 1.f - ps;
        if (!specular) *proportional = true;
        return true;
    }
    float pdf = full_pdf(b, wo, s->wi);
    if (pdf == 0.f) return false;
    s->f = full_f(b, wo, s->wi);
    s->pdf = pdf;
    return true;
}

} // namespace prb
