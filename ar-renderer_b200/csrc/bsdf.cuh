// Surface scattering on the device: Lambertian reflection, anisotropic Trowbridge-Reitz (GGX)
// conductors with spectral complex Fresnel, and smooth / rough / thin dielectrics, each with
// f, pdf and importance sampling in the local shading frame (z = normal). These are the pbrt-v4
// models the reference implements in src/materials/bxdf.cpp:19-256 (microfacet distribution
// bxdf.h:76-115); results agree with them to float rounding on identical inputs.
#pragma once

#include "common.cuh"

namespace prb {

enum : uint32_t { kFlagReflection = 1, kFlagTransmission = 2, kFlagDiffuse = 4, kFlagGlossy = 8, kFlagSpecular = 16 };
enum : int { kLobeDiffuse = 0, kLobeConductor = 1, kLobeDielectric = 2, kLobeThin = 3, kLobeNone = 4 };
// Which scattering kinds a sample or pdf may use (pbrt-v4's BxDFReflTransFlags).
enum : int { kSampleR = 1, kSampleT = 2, kSampleAll = 3 };

// Trowbridge-Reitz microfacet distribution with the visible-normal sampling of Heitz (2018).
struct Ggx {
    float ax, ay;
    __device__ bool smooth() const { return fmaxf(ax, ay) < 1e-3f; }
    __device__ static float cos2(V3 w) { return w.z * w.z; }
    __device__ static float sin2(V3 w) { return fmaxf(0.f, 1.f - cos2(w)); }
    __device__ static float tan2(V3 w) { return sin2(w) / cos2(w); }
    __device__ static float cos_phi(V3 w) {
        float s = safe_sqrt(sin2(w));
        return s == 0.f ? 1.f : clampf(w.x / s, -1.f, 1.f);
    }
    __device__ static float sin_phi(V3 w) {
        float s = safe_sqrt(sin2(w));
        return s == 0.f ? 0.f : clampf(w.y / s, -1.f, 1.f);
    }
    __device__ float D(V3 wm) const {
        float t2 = tan2(wm);
        if (isinf(t2)) return 0.f;
        float c4 = sqr(cos2(wm));
        if (c4 < 1e-16f) return 0.f;
        float e = t2 * (sqr(cos_phi(wm) / ax) + sqr(sin_phi(wm) / ay));
        return 1.f / (kPi * ax * ay * c4 * sqr(1.f + e));
    }
    __device__ float lambda(V3 w) const {
        float t2 = tan2(w);
        if (isinf(t2)) return 0.f;
        float a2 = sqr(cos_phi(w) * ax) + sqr(sin_phi(w) * ay);
        return (sqrtf(1.f + a2 * t2) - 1.f) * 0.5f;
    }
    __device__ float G1(V3 w) const { return 1.f / (1.f + lambda(w)); }
    __device__ float G(V3 wo, V3 wi) const { return 1.f / (1.f + lambda(wo) + lambda(wi)); }
    // Density of visible normals wm seen from w.
    __device__ float pdf(V3 w, V3 wm) const { return G1(w) / fabsf(w.z) * D(wm) * fabsf(dot(w, wm)); }
    __device__ V3 sample_wm(V3 w, float u0, float u1) const {
        V3 wh = normalize(mk(ax * w.x, ay * w.y, w.z));
        if (wh.z < 0.f) wh = -wh;
        V3 t1 = wh.z < 0.99999f ? normalize(cross(mk(0.f, 0.f, 1.f), wh)) : mk(1.f, 0.f, 0.f);
        V3 t2 = cross(wh, t1);
        float r = sqrtf(u0), phi = 2.f * kPi * u1;
        float sp, cp;
        sincos_rn(phi, &sp, &cp);
        float px = r * cp, py = r * sp;
        float h = sqrtf(1.f - px * px);
        float s = (1.f + wh.z) * 0.5f;
        py = (1.f - s) * h + s * py;
        float pz = sqrtf(fmaxf(0.f, 1.f - px * px - py * py));
        V3 nh = t1 * px + t2 * py + wh * pz;
        return normalize(mk(ax * nh.x, ay * nh.y, fmaxf(1e-6f, nh.z)));
    }
};

// Unpolarised Fresnel reflectance of a dielectric interface (eta = transmitted / incident IOR).
__device__ __forceinline__ float fr_dielectric(float cosI, float eta) {
    cosI = clampf(cosI, -1.f, 1.f);
    if (cosI < 0.f) {
        eta = 1.f / eta;
        cosI = -cosI;
    }
    float sin2T = (1.f - sqr(cosI)) / sqr(eta);
    if (sin2T >= 1.f) return 1.f;
    float cosT = safe_sqrt(1.f - sin2T);
    float rpa = (eta * cosI - cosT) / (eta * cosI + cosT);
    float rpe = (cosI - eta * cosT) / (cosI + eta * cosT);
    return (sqr(rpa) + sqr(rpe)) * 0.5f;
}

// Fresnel reflectance of a conductor with complex IOR eta + i k, in explicit complex arithmetic.
struct Cpx {
    float re, im;
};
__device__ __forceinline__ Cpx cmul(Cpx a, Cpx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ Cpx cdiv(Cpx a, Cpx b) {
    float d = b.re * b.re + b.im * b.im;
    return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
__device__ __forceinline__ Cpx csqrt(Cpx z) {
    // Principal root in the algebraic form (no trigonometry): with h = |z|,
    // re = sqrt((h + x) / 2), im = y / (2 re) for x >= 0, and the mirrored form for x < 0.
    if (z.re == 0.f && z.im == 0.f) return {0.f, z.im};
    float h = hypotf(z.re, z.im);
    if (z.re > 0.f) {
        float d = sqrtf(0.5f * (h + z.re));
        return {d, 0.5f * (z.im / d)};
    }
    float s = sqrtf(0.5f * (h - z.re));
    return {fabsf(0.5f * (z.im / s)), copysignf(s, z.im)};
}
__device__ __forceinline__ float fr_complex(float cosI, float etaR, float etaI) {
    cosI = clampf(cosI, 0.f, 1.f);
    float sin2I = 1.f - sqr(cosI);
    Cpx eta{etaR, etaI};
    Cpx sin2T = cdiv(Cpx{sin2I, 0.f}, cmul(eta, eta));
    Cpx cosT = csqrt(Cpx{1.f - sin2T.re, -sin2T.im});
    Cpx ec{eta.re * cosI, eta.im * cosI};
    Cpx rpa = cdiv(Cpx{ec.re - cosT.re, ec.im - cosT.im}, Cpx{ec.re + cosT.re, ec.im + cosT.im});
    Cpx ect = cmul(eta, cosT);
    Cpx rpe = cdiv(Cpx{cosI - ect.re, -ect.im}, Cpx{cosI + ect.re, ect.im});
    return (rpa.re * rpa.re + rpa.im * rpa.im + rpe.re * rpe.re + rpe.im * rpe.im) * 0.5f;
}

// Refraction of wi about n with relative IOR eta; false on total internal reflection.
__device__ __forceinline__ bool refract(V3 wi, V3 n, float eta, float *etap, V3 *wt) {
    float cosI = dot(n, wi);
    if (cosI < 0.f) {
        eta = 1.f / eta;
        cosI = -cosI;
        n = -n;
    }
    float sin2I = fmaxf(0.f, 1.f - sqr(cosI));
    float sin2T = sin2I / sqr(eta);
    if (sin2T >= 1.f) return false;
    float cosT = safe_sqrt(1.f - sin2T);
    *wt = -wi * (1.f / eta) + n * (cosI / eta - cosT);
    *etap = eta;
    return true;
}

__device__ __forceinline__ bool same_hemi(V3 a, V3 b) { return a.z * b.z > 0.f; }

// Concentric disk mapping (Shirley-Chiu) and the cosine-weighted hemisphere built on it.
__device__ __forceinline__ void concentric_disk(float u0, float u1, float *x, float *y) {
    float ox = 2.f * u0 - 1.f, oy = 2.f * u1 - 1.f;
    if (ox == 0.f && oy == 0.f) {
        *x = *y = 0.f;
        return;
    }
    float r, th;
    if (fabsf(ox) > fabsf(oy)) {
        r = ox;
        th = kPiOver4 * (oy / ox);
    } else {
        r = oy;
        th = kPiOver2 - kPiOver4 * (ox / oy);
    }
    float s, c;
    sincos_rn(th, &s, &c);
    *x = r * c;
    *y = r * s;
}
__device__ __forceinline__ V3 cosine_hemisphere(float u0, float u1) {
    float x, y;
    concentric_disk(u0, u1, &x, &y);
    return mk(x, y, safe_sqrt(1.f - x * x - y * y));
}

// One BxDF with its parameters at the 4 sampled wavelengths.
struct Lobe {
    int kind;
    SS R;          // diffuse reflectance
    SS eta, k;     // conductor
    float etaD;    // dielectric / thin IOR at the hero wavelength
    Ggx mf;
    __device__ bool specular() const {
        switch (kind) {
        case kLobeDiffuse: return false;
        case kLobeThin: return true;
        case kLobeNone: return true;
        default: return mf.smooth();
        }
    }
    __device__ uint32_t flags() const {
        switch (kind) {
        case kLobeDiffuse: return nonzero(R) ? (kFlagReflection | kFlagDiffuse) : 0u;
        case kLobeConductor: return kFlagReflection | (mf.smooth() ? kFlagSpecular : kFlagGlossy);
        case kLobeDielectric:
            return (etaD == 1.f ? kFlagTransmission : (kFlagReflection | kFlagTransmission)) |
                   (mf.smooth() ? kFlagSpecular : kFlagGlossy);
        case kLobeThin: return kFlagReflection | kFlagTransmission | kFlagSpecular;
        default: return 0u;
        }
    }
    // True when the lobe has a diffuse or glossy component (next-event estimation applies).
    __device__ bool non_specular() const { return (flags() & (kFlagDiffuse | kFlagGlossy)) != 0u; }
};

struct BSample {
    SS f;
    V3 wi;
    float pdf;
    uint32_t flags;
    float eta;
};

__device__ __forceinline__ SS conductor_f(const Lobe &l, V3 wo, V3 wi) {
    if (!same_hemi(wo, wi) || l.mf.smooth()) return splat(0.f);
    float co = fabsf(wo.z), ci = fabsf(wi.z);
    if (ci == 0.f || co == 0.f) return splat(0.f);
    V3 wm = wi + wo;
    if (len2(wm) == 0.f) return splat(0.f);
    wm = normalize(wm);
    float c = fabsf(dot(wo, wm));
    float d = l.mf.D(wm) * l.mf.G(wo, wi) / (4.f * ci * co);
    SS F;
#pragma unroll
    for (int i = 0; i < 4; ++i) F.v[i] = fr_complex(c, l.eta.v[i], l.k.v[i]) * d;
    return F;
}

// radiance = true: radiance transport (1/eta^2 scaling of transmission).
__device__ __forceinline__ float dielectric_f(const Lobe &l, V3 wo, V3 wi, bool radiance) {
    if (l.etaD == 1.f || l.mf.smooth()) return 0.f;
    float co = wo.z, ci = wi.z;
    bool refl = ci * co > 0.f;
    float etap = 1.f;
    if (!refl) etap = co > 0.f ? l.etaD : 1.f / l.etaD;
    V3 wm = wi * etap + wo;
    if (ci == 0.f || co == 0.f || len2(wm) == 0.f) return 0.f;
    wm = face_forward(normalize(wm), mk(0.f, 0.f, 1.f));
    if (dot(wm, wi) * ci < 0.f || dot(wm, wo) * co < 0.f) return 0.f;
    float F = fr_dielectric(dot(wo, wm), l.etaD);
    if (refl) return l.mf.D(wm) * l.mf.G(wo, wi) * F / fabsf(4.f * ci * co);
    float denom = sqr(dot(wi, wm) + dot(wo, wm) / etap) * ci * co;
    float ft = l.mf.D(wm) * (1.f - F) * l.mf.G(wo, wi) * fabsf(dot(wi, wm) * dot(wo, wm) / denom);
    return radiance ? ft / sqr(etap) : ft;
}

__device__ __forceinline__ float dielectric_pdf(const Lobe &l, V3 wo, V3 wi, int mode = kSampleAll) {
    if (l.etaD == 1.f || l.mf.smooth()) return 0.f;
    float co = wo.z, ci = wi.z;
    bool refl = ci * co > 0.f;
    float etap = 1.f;
    if (!refl) etap = co > 0.f ? l.etaD : 1.f / l.etaD;
    V3 wm = wi * etap + wo;
    if (ci == 0.f || co == 0.f || len2(wm) == 0.f) return 0.f;
    wm = face_forward(normalize(wm), mk(0.f, 0.f, 1.f));
    if (dot(wm, wi) * ci < 0.f || dot(wm, wo) * co < 0.f) return 0.f;
    float R = fr_dielectric(dot(wo, wm), l.etaD), T = 1.f - R;
    if (!(mode & kSampleR)) R = 0.f;
    if (!(mode & kSampleT)) T = 0.f;
    if (R == 0.f && T == 0.f) return 0.f;
    if (refl) return l.mf.pdf(wo, wm) / (4.f * fabsf(dot(wo, wm))) * R / (R + T);
    float denom = sqr(dot(wi, wm) + dot(wo, wm) / etap);
    return l.mf.pdf(wo, wm) * fabsf(dot(wi, wm)) / denom * T / (R + T);
}

__device__ __forceinline__ SS lobe_f(const Lobe &l, V3 wo, V3 wi, bool radiance = true) {
    switch (l.kind) {
    case kLobeDiffuse: return same_hemi(wo, wi) ? l.R * kInvPi : splat(0.f);
    case kLobeConductor: return conductor_f(l, wo, wi);
    case kLobeDielectric: return splat(dielectric_f(l, wo, wi, radiance));
    default: return splat(0.f);
    }
}

// mode: the scattering kinds the matching sample may use (kSampleAll in the path tracer; the
// layered walks restrict interfaces to reflection or transmission).
__device__ __forceinline__ float lobe_pdf(const Lobe &l, V3 wo, V3 wi, int mode = kSampleAll) {
    switch (l.kind) {
    case kLobeDiffuse: return (mode & kSampleR) && same_hemi(wo, wi) ? fabsf(wi.z) * kInvPi : 0.f;
    case kLobeConductor: {
        if (!(mode & kSampleR) || !same_hemi(wo, wi) || l.mf.smooth()) return 0.f;
        V3 wm = wo + wi;
        if (len2(wm) == 0.f) return 0.f;
        wm = face_forward(normalize(wm), mk(0.f, 0.f, 1.f));
        return l.mf.pdf(wo, wm) / (4.f * fabsf(dot(wo, wm)));
    }
    case kLobeDielectric: return dielectric_pdf(l, wo, wi, mode);
    default: return 0.f;
    }
}

// Importance sampling; false when no direction is produced.
__device__ __forceinline__ bool lobe_sample(const Lobe &l, V3 wo, float uc, float u0, float u1, BSample *s,
                                            bool radiance = true, int mode = kSampleAll) {
    s->eta = 1.f;
    if ((l.kind == kLobeDiffuse || l.kind == kLobeConductor) && !(mode & kSampleR)) return false;
    switch (l.kind) {
    case kLobeDiffuse: {
        V3 wi = cosine_hemisphere(u0, u1);
        if (wo.z < 0.f) wi.z = -wi.z;
        s->wi = wi;
        s->pdf = fabsf(wi.z) * kInvPi;
        s->f = l.R * kInvPi;
        s->flags = kFlagReflection | kFlagDiffuse;
        return true;
    }
    case kLobeConductor: {
        if (l.mf.smooth()) {
            V3 wi = mk(-wo.x, -wo.y, wo.z);
            float c = fabsf(wi.z);
#pragma unroll
            for (int i = 0; i < 4; ++i) s->f.v[i] = fr_complex(c, l.eta.v[i], l.k.v[i]) / c;
            s->wi = wi;
            s->pdf = 1.f;
            s->flags = kFlagReflection | kFlagSpecular;
            return true;
        }
        if (wo.z == 0.f) return false;
        V3 wm = l.mf.sample_wm(wo, u0, u1);
        V3 wi = -wo + wm * (2.f * dot(wo, wm));
        if (!same_hemi(wo, wi)) return false;
        float co = fabsf(wo.z), ci = fabsf(wi.z);
        if (ci == 0.f || co == 0.f) return false;
        s->pdf = l.mf.pdf(wo, wm) / (4.f * fabsf(dot(wo, wm)));
        float c = fabsf(dot(wo, wm));
        float d = l.mf.D(wm) * l.mf.G(wo, wi) / (4.f * ci * co);
#pragma unroll
        for (int i = 0; i < 4; ++i) s->f.v[i] = fr_complex(c, l.eta.v[i], l.k.v[i]) * d;
        s->wi = wi;
        s->flags = kFlagReflection | kFlagGlossy;
        return true;
    }
    case kLobeThin: {
        float R = fr_dielectric(fabsf(wo.z), l.etaD), T = 1.f - R;
        if (R < 1.f) {
            // Interreflection inside the slab (geometric series).
            R += sqr(T) * R / (1.f - sqr(R));
            T = 1.f - R;
        }
        if (!(mode & kSampleR)) R = 0.f;
        if (!(mode & kSampleT)) T = 0.f;
        if (R == 0.f && T == 0.f) return false;
        if (uc < R / (R + T)) {
            V3 wi = mk(-wo.x, -wo.y, wo.z);
            s->f = splat(R / fabsf(wi.z));
            s->pdf = R / (R + T);
            s->wi = wi;
            s->flags = kFlagReflection | kFlagSpecular;
        } else {
            V3 wi = -wo;
            s->f = splat(T / fabsf(wi.z));
            s->pdf = T / (R + T);
            s->wi = wi;
            s->flags = kFlagTransmission | kFlagSpecular;
        }
        return true;
    }
    case kLobeDielectric: {
        if (l.etaD == 1.f || l.mf.smooth()) {
            float R = fr_dielectric(wo.z, l.etaD), T = 1.f - R;
            if (!(mode & kSampleR)) R = 0.f;
            if (!(mode & kSampleT)) T = 0.f;
            if (R == 0.f && T == 0.f) return false;
            if (uc < R / (R + T)) {
                V3 wi = mk(-wo.x, -wo.y, wo.z);
                s->f = splat(R / fabsf(wi.z));
                s->pdf = R / (R + T);
                s->wi = wi;
                s->flags = kFlagReflection | kFlagSpecular;
                return true;
            }
            V3 wi;
            float etap;
            if (!refract(wo, mk(0.f, 0.f, 1.f), l.etaD, &etap, &wi)) return false;
            float ft = T / fabsf(wi.z);
            s->f = splat(radiance ? ft / sqr(etap) : ft);
            s->pdf = T / (R + T);
            s->wi = wi;
            s->flags = kFlagTransmission | kFlagSpecular;
            s->eta = etap;
            return true;
        }
        V3 wm = l.mf.sample_wm(wo, u0, u1);
        float R = fr_dielectric(dot(wo, wm), l.etaD), T = 1.f - R;
        if (!(mode & kSampleR)) R = 0.f;
        if (!(mode & kSampleT)) T = 0.f;
        if (R == 0.f && T == 0.f) return false;
        if (uc < R / (R + T)) {
            V3 wi = -wo + wm * (2.f * dot(wo, wm));
            if (!same_hemi(wo, wi)) return false;
            s->pdf = l.mf.pdf(wo, wm) / (4.f * fabsf(dot(wo, wm))) * R / (R + T);
            s->f = splat(l.mf.D(wm) * l.mf.G(wo, wi) * R / (4.f * wi.z * wo.z));
            s->wi = wi;
            s->flags = kFlagReflection | kFlagGlossy;
            return true;
        }
        V3 wi;
        float etap;
        if (!refract(wo, wm, l.etaD, &etap, &wi) || same_hemi(wo, wi) || wi.z == 0.f) return false;
        float denom = sqr(dot(wi, wm) + dot(wo, wm) / etap);
        s->pdf = l.mf.pdf(wo, wm) * fabsf(dot(wi, wm)) / denom * T / (R + T);
        float ft = T * l.mf.D(wm) * l.mf.G(wo, wi) * fabsf(dot(wi, wm) * dot(wo, wm) / (wi.z * wo.z * denom));
        s->f = splat(radiance ? ft / sqr(etap) : ft);
        s->wi = wi;
        s->flags = kFlagTransmission | kFlagGlossy;
        s->eta = etap;
        return true;
    }
    default: return false;
    }
}

// Henyey-Greenstein phase function and its exact sampling (p / pdf = 1).
__device__ __forceinline__ float hg_phase(float cosTheta, float g) {
    float denom = 1.f + sqr(g) + 2.f * g * cosTheta;
    return kInv4Pi * (1.f - sqr(g)) / (denom * safe_sqrt(denom));
}
__device__ __forceinline__ V3 hg_sample(V3 wo, float g, float u0, float u1, float *pdf) {
    float cosTheta;
    if (fabsf(g) < 1e-3f)
        cosTheta = 1.f - 2.f * u0;
    else
        cosTheta = -1.f / (2.f * g) * (1.f + sqr(g) - sqr((1.f - sqr(g)) / (1.f + g - 2.f * g * u0)));
    cosTheta = clampf(cosTheta, -1.f, 1.f);
    float sinTheta = safe_sqrt(1.f - sqr(cosTheta));
    float s, c;
    sincos_rn(2.f * kPi * u1, &s, &c);
    Frame f = frame_from_z(wo);
    *pdf = hg_phase(cosTheta, g);
    return f.from_local(mk(sinTheta * c, sinTheta * s, cosTheta));
}

} // namespace prb
