// Oracle harness: a C ABI over the reference renderer's own CPU code (PRender, compiled from its
// sources by oracle/Makefile into oracle/_ref/). This file is TEST INFRASTRUCTURE: only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm load it, as the checker or
// as the timed CPU reference -- never as the thing measured or shipped.
//
// Everything here calls the reference's public C++ API unchanged:
//   BVH::Build / Intersect / IntersectP          src/geometry/bvh.cpp:8-232
//   Triangle::Intersect                          src/geometry/shape.cpp:202-222
//   DiffuseBxDF / ConductorBxDF / DielectricBxDF / ThinDielectricBxDF  src/materials/bxdf.cpp:85-256
//   HenyeyGreenstein / SampleHenyeyGreenstein     src/materials/bxdf.cpp:64-80
//   HomogeneousMedium::Transmittance / SampleDistanceHero  src/media/medium.cpp:15-103
//   SampledWavelengths::SampleVisible, CIE_X/Y/Z  src/core/spectrum.cpp:32-66
//   LoadScene + PathIntegrator::Render           src/scene/scene_loader.cpp:1364, src/integrators/path.cpp:51-80
//   BVHLightSampler::Sample / PMF                src/lights/light_bvh.cpp:179-234
// The scene exporter below restates the flattening that src/integrators/gpu_path.cpp:108-456 does
// before it calls prgpu_render, so the CUDA module receives exactly what the reference host would
// hand its GPU module.

#include "cameras/camera.h"
#include "core/color.h"
#include "core/film.h"
#include "core/parallel.h"
#include "core/rgb2spec.h"
#include "core/serialize.h"
#include "core/spectrum.h"
#include "geometry/bvh.h"
#include "geometry/shape.h"
#include "gpu/gpu_api.h"
#include "integrators/aov.h"
#include "integrators/integrator.h"
#include "integrators/path.h"
#include "lights/light.h"
#include "lights/light_bvh.h"
#include "materials/bxdf.h"
#include "materials/material.h"
#include "materials/texture.h"
#include "media/medium.h"
#include "scene/scene.h"
#include "scene/scene_loader.h"

#include <chrono>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

using namespace pr;

#define API extern "C" __attribute__((visibility("default")))

namespace {

void SetErr(char *err, int len, const std::string &m) {
    if (err && len > 0) std::snprintf(err, size_t(len), "%s", m.c_str());
}

struct SoupBVH {
    std::shared_ptr<TriangleMesh> mesh;
    std::vector<std::unique_ptr<Triangle>> tris;
    BVH bvh;
};

} // namespace

// ---------------------------------------------------------------------------------------------
// Threads and the RGB->spectrum table cache

API void prref_set_threads(int n) { SetThreadCount(n); }
API int prref_thread_count() { return ThreadCount(); }
API void prref_set_cache_dir(const char *dir) { RGBToSpectrumTable::SetCacheDirectory(dir); }

// ---------------------------------------------------------------------------------------------
// Triangle-soup BVH (traversal microbenchmark and bit-exact traversal parity)

// verts: n triangles x 9 floats (p0, p1, p2). Builds the reference's binned-SAH BVH.
API void *prref_soup_new(const float *verts, int64_t n) {
    auto *s = new SoupBVH;
    s->mesh = std::make_shared<TriangleMesh>();
    s->mesh->p.resize(size_t(3 * n));
    s->mesh->indices.resize(size_t(3 * n));
    for (int64_t i = 0; i < 3 * n; ++i) {
        s->mesh->p[size_t(i)] = Vec3f(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]);
        s->mesh->indices[size_t(i)] = int(i);
    }
    std::vector<const Shape *> shapes;
    shapes.reserve(size_t(n));
    s->tris.reserve(size_t(n));
    for (int64_t t = 0; t < n; ++t) {
        s->tris.push_back(std::make_unique<Triangle>(s->mesh, int(t)));
        shapes.push_back(s->tris.back().get());
    }
    s->bvh.Build(std::move(shapes));
    return s;
}

API void prref_soup_free(void *h) { delete static_cast<SoupBVH *>(h); }

API int64_t prref_soup_node_count(void *h) { return int64_t(static_cast<SoupBVH *>(h)->bvh.Nodes().size()); }

// Exports the flattened nodes in the prgpu::BVHNode layout (as gpu_path.cpp:378-390 does) and the
// leaf-slot -> triangle permutation.
API void prref_soup_export(void *h, prgpu::BVHNode *nodes, int32_t *order) {
    const BVH &b = static_cast<SoupBVH *>(h)->bvh;
    const auto &ns = b.Nodes();
    for (size_t i = 0; i < ns.size(); ++i) {
        prgpu::BVHNode g{};
        g.bmin = {ns[i].bounds.pMin.x, ns[i].bounds.pMin.y, ns[i].bounds.pMin.z};
        g.bmax = {ns[i].bounds.pMax.x, ns[i].bounds.pMax.y, ns[i].bounds.pMax.z};
        g.offset = ns[i].offset;
        g.nPrims = ns[i].nPrims;
        g.axis = ns[i].axis;
        nodes[i] = g;
    }
    const auto &o = b.Order();
    for (size_t i = 0; i < o.size(); ++i) order[i] = o[i];
}

// rays: n x 8 floats (ox, oy, oz, dx, dy, dz, tmax, unused). Closest hit writes prim (original
// index, -1 = miss), t, b1, b2; any-hit writes prim = 1/0. Runs under the reference ParallelFor.
// Returns the wall time in seconds.
API double prref_soup_trace(void *h, const float *rays, int64_t n, int anyHit, int32_t *prim, float *t, float *b1,
                            float *b2) {
    const BVH &bvh = static_cast<SoupBVH *>(h)->bvh;
    auto t0 = std::chrono::steady_clock::now();
    ParallelFor(
        n,
        [&](int64_t i, int) {
            const float *r = rays + 8 * i;
            Ray ray(Vec3f(r[0], r[1], r[2]), Vec3f(r[3], r[4], r[5]));
            if (anyHit) {
                prim[i] = bvh.IntersectP(ray, r[6]) ? 1 : 0;
                return;
            }
            BVH::Hit hit;
            if (bvh.Intersect(ray, r[6], &hit)) {
                prim[i] = hit.prim;
                if (t) t[i] = hit.t;
                if (b1) b1[i] = hit.info.b1;
                if (b2) b2[i] = hit.info.b2;
            } else {
                prim[i] = -1;
                if (t) t[i] = 0;
                if (b1) b1[i] = 0;
                if (b2) b2[i] = 0;
            }
        },
        1024);
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// ---------------------------------------------------------------------------------------------
// BxDFs on identical local-frame inputs
//
// kind: 0 diffuse, 1 conductor, 2 dielectric, 3 thin dielectric.
// params (16 floats): R[4] | eta[4] | k[4] | etaD, alphaX, alphaY, mode(0 radiance, 1 importance)
// in  (per item, 9 floats): wo[3], wi[3], uc, u0, u1
// out (per item, 16 floats): f[4], pdf, sample: ok, f[4], pdf, wi[3], flags, eta
API void prref_bxdf(int kind, const float *params, int64_t n, const float *in, float *out) {
    SampledSpectrum R, eta, k;
    for (int i = 0; i < 4; ++i) {
        R[i] = params[i];
        eta[i] = params[4 + i];
        k[i] = params[8 + i];
    }
    float etaD = params[12];
    TrowbridgeReitzDistribution distrib(params[13], params[14]);
    TransportMode mode = params[15] != 0 ? TransportMode::Importance : TransportMode::Radiance;
    DiffuseBxDF diffuse(R);
    ConductorBxDF conductor(distrib, eta, k);
    DielectricBxDF dielectric(etaD, distrib);
    ThinDielectricBxDF thin(etaD);
    const BxDF *bxdf = kind == 0 ? static_cast<const BxDF *>(&diffuse)
                       : kind == 1 ? static_cast<const BxDF *>(&conductor)
                       : kind == 2 ? static_cast<const BxDF *>(&dielectric)
                                   : static_cast<const BxDF *>(&thin);
    for (int64_t j = 0; j < n; ++j) {
        const float *x = in + 9 * j;
        float *y = out + 16 * j;
        Vec3f wo(x[0], x[1], x[2]), wi(x[3], x[4], x[5]);
        SampledSpectrum f = bxdf->f(wo, wi, mode);
        for (int i = 0; i < 4; ++i) y[i] = f[i];
        y[4] = bxdf->PDF(wo, wi, mode, BxDFReflTransFlags::All);
        auto bs = bxdf->Sample_f(wo, x[6], Vec2f(x[7], x[8]), mode, BxDFReflTransFlags::All);
        std::memset(y + 5, 0, 11 * sizeof(float));
        if (bs) {
            y[5] = 1;
            for (int i = 0; i < 4; ++i) y[6 + i] = bs->f[i];
            y[10] = bs->pdf;
            y[11] = bs->wi.x;
            y[12] = bs->wi.y;
            y[13] = bs->wi.z;
            y[14] = float(uint32_t(bs->flags));
            y[15] = bs->eta;
        }
    }
}

// Coated / sheen BxDFs on identical local-frame inputs: pr::LayeredBxDF (dielectric coat over a
// diffuse or conductor base, two-sided) and pr::SheenBxDF over it or over a single lobe.
// params (36 floats): layered, base kind (0 diffuse, 1 conductor, 2 dielectric), R[4], eta[4],
//   k[4], etaD, alphaX, alphaY, coat eta, coat alpha, thickness, g, albedo[4], maxDepth,
//   nSamples, sheen weight, sheen roughness, sheen colour[4], 2 unused
// in (9 floats): wo[3], wi[3], uc, u0, u1
// out (16 floats): f[4], pdf, sample: ok, f[4], pdf, wi[3], flags, pdf-is-proportional
API void prref_full_bsdf(const float *params, int64_t n, const float *in, float *out) {
    auto ss = [&](int o) {
        SampledSpectrum v;
        for (int i = 0; i < 4; ++i) v[i] = params[o + i];
        return v;
    };
    const bool layered = params[0] != 0;
    const int kind = int(params[1]);
    TrowbridgeReitzDistribution baseMf(params[15], params[16]);
    DiffuseBxDF diffuse(ss(2));
    ConductorBxDF conductor(baseMf, ss(6), ss(10));
    DielectricBxDF dielectric(params[14], baseMf);
    const BxDF *base = kind == 0 ? static_cast<const BxDF *>(&diffuse)
                       : kind == 1 ? static_cast<const BxDF *>(&conductor)
                                   : static_cast<const BxDF *>(&dielectric);
    DielectricBxDF coat(params[17], TrowbridgeReitzDistribution(params[18], params[18]));
    LayeredBxDF lay(&coat, base, params[19], ss(21), params[20], true, int(params[25]), int(params[26]));
    const BxDF *b = layered ? static_cast<const BxDF *>(&lay) : base;
    SheenBxDF sheen(b, ss(29), params[28], params[27]);
    if (params[27] > 0) b = &sheen;
    for (int64_t j = 0; j < n; ++j) {
        const float *x = in + 9 * j;
        float *y = out + 16 * j;
        Vec3f wo(x[0], x[1], x[2]), wi(x[3], x[4], x[5]);
        SampledSpectrum f = b->f(wo, wi, TransportMode::Radiance);
        for (int i = 0; i < 4; ++i) y[i] = f[i];
        y[4] = b->PDF(wo, wi, TransportMode::Radiance, BxDFReflTransFlags::All);
        auto bs = b->Sample_f(wo, x[6], Vec2f(x[7], x[8]), TransportMode::Radiance, BxDFReflTransFlags::All);
        std::memset(y + 5, 0, 11 * sizeof(float));
        if (bs) {
            y[5] = 1;
            for (int i = 0; i < 4; ++i) y[6 + i] = bs->f[i];
            y[10] = bs->pdf;
            y[11] = bs->wi.x;
            y[12] = bs->wi.y;
            y[13] = bs->wi.z;
            y[14] = float(uint32_t(bs->flags));
            y[15] = bs->pdfIsProportional ? 1.f : 0.f;
        }
    }
}

// Checkpoints through the reference's own WriteCheckpoint / ReadCheckpoint (integrator.cpp:30-90)
// for a path-tracer render (body: the samples per pixel as int32). The film's accumulators are set
// exactly through Film::ReadAccumulators from a scratch file (AddPixelXYZ takes floats).
static void checkpoint_setup(RenderControl *c, IntegratorSettings *s, uint64_t fingerprint, uint64_t seed, int device,
                             int maxDepth) {
    c->fingerprint = fingerprint;
    c->seed = seed;
    s->type = IntegratorType::Path;
    s->device = device;
    s->maxDepth = maxDepth;
}

API int prref_checkpoint_write(const char *path, int width, int height, int device, int maxDepth, uint64_t fingerprint,
                               uint64_t seed, const double *film, int32_t passes, char *err, int errLen) {
    FilmSettings fs;
    fs.width = width;
    fs.height = height;
    Film f(fs);
    std::string scratch = std::string(path) + ".acc";
    FILE *t = std::fopen(scratch.c_str(), "wb");
    uint64_t n = uint64_t(width) * height * 3;
    bool ok = t && std::fwrite(&n, sizeof(n), 1, t) == 1 && std::fwrite(film, sizeof(double), n, t) == n;
    if (t) std::fclose(t);
    t = ok ? std::fopen(scratch.c_str(), "rb") : nullptr;
    ok = t && f.ReadAccumulators(t);
    if (t) std::fclose(t);
    std::remove(scratch.c_str());
    RenderControl c;
    IntegratorSettings s;
    c.checkpointPath = path;
    checkpoint_setup(&c, &s, fingerprint, seed, device, maxDepth);
    std::string e;
    ok = ok && WriteCheckpoint(c, s, f, [&](BinaryWriter &w) { w.Put(int32_t(passes)); }, &e);
    if (!ok) std::snprintf(err, size_t(errLen), "%s", e.c_str());
    return ok ? 0 : 1;
}

API int prref_checkpoint_read(const char *path, int width, int height, int device, int maxDepth, uint64_t fingerprint,
                              uint64_t seed, double *film, int32_t *passes, char *err, int errLen) {
    FilmSettings fs;
    fs.width = width;
    fs.height = height;
    Film f(fs);
    RenderControl c;
    IntegratorSettings s;
    c.resumePath = path;
    checkpoint_setup(&c, &s, fingerprint, seed, device, maxDepth);
    std::string e;
    if (!ReadCheckpoint(c, s, f, [&](BinaryReader &r) { return r.Get(passes); }, &e)) {
        std::snprintf(err, size_t(errLen), "%s", e.c_str());
        return 1;
    }
    // The accumulators leave through a scratch file (PixelXYZ rounds them to float).
    std::string scratch = std::string(path) + ".acc";
    FILE *t = std::fopen(scratch.c_str(), "wb");
    bool ok = t && f.WriteAccumulators(t);
    if (t) std::fclose(t);
    t = ok ? std::fopen(scratch.c_str(), "rb") : nullptr;
    uint64_t n = 0;
    ok = t && std::fread(&n, sizeof(n), 1, t) == 1 && n == uint64_t(width) * height * 3 &&
         std::fread(film, sizeof(double), n, t) == n;
    if (t) std::fclose(t);
    std::remove(scratch.c_str());
    return ok ? 0 : 1;
}

// The sheen lobe's directional albedo at the table nodes ([16 roughness][32 cos theta]).
API void prref_sheen_table(float *out) {
    for (int ia = 0; ia < prgpu::kSheenAlpha; ++ia)
        for (int im = 0; im < prgpu::kSheenMu; ++im)
            out[ia * prgpu::kSheenMu + im] =
                SheenBxDF::Albedo(float(im) / (prgpu::kSheenMu - 1), 0.05f + 0.95f * float(ia) / (prgpu::kSheenAlpha - 1));
}

// Scalar Fresnel terms (known-answer tests): FrDielectric and FrComplex (per wavelength).
API float prref_fr_dielectric(float cosI, float eta) { return FrDielectric(cosI, eta); }
API float prref_fr_complex(float cosI, float eta, float k) {
    return FrComplex(cosI, SampledSpectrum(eta), SampledSpectrum(k))[0];
}

// Henyey-Greenstein: in (per item, 7 floats) cosTheta, g, wo[3], u0, u1
// out (per item, 5 floats): p(cosTheta, g), wi[3], pdf of the sampled direction
API void prref_hg(int64_t n, const float *in, float *out) {
    for (int64_t j = 0; j < n; ++j) {
        const float *x = in + 7 * j;
        float *y = out + 5 * j;
        y[0] = HenyeyGreenstein(x[0], x[1]);
        float pdf = 0;
        Vec3f wi = SampleHenyeyGreenstein(Vec3f(x[2], x[3], x[4]), x[1], Vec2f(x[5], x[6]), &pdf);
        y[1] = wi.x;
        y[2] = wi.y;
        y[3] = wi.z;
        y[4] = pdf;
    }
}

// Homogeneous medium with constant-per-wavelength sigma_a, sigma_s given at the 4 sampled
// wavelengths (the caller tabulates them). in (per item, 10 floats): sa[4], ss[4], tMax, u.
// out (per item, 14 floats): Tr(tMax)[4], scattered, t, weight[4], pdfRatio[4].
namespace {
struct Sampled4Spectrum : Spectrum {
    float v[4];
    float l[4];
    float operator()(float lambda) const override {
        for (int i = 0; i < 4; ++i)
            if (lambda == l[i]) return v[i];
        return 0;
    }
    float MaxValue() const override { return std::max(std::max(v[0], v[1]), std::max(v[2], v[3])); }
};
} // namespace

API void prref_homogeneous(int64_t n, const float *lambda4, const float *in, float *out) {
    // Wavelengths fixed for the batch so that Spectrum::Sample picks the given per-lambda values.
    SampledWavelengths swl = SampledWavelengths::SampleVisible(0.37f);
    float lam[4];
    for (int i = 0; i < 4; ++i) lam[i] = swl[i];
    for (int64_t j = 0; j < n; ++j) {
        const float *x = in + 10 * j;
        float *y = out + 14 * j;
        auto sa = std::make_shared<Sampled4Spectrum>(), ss = std::make_shared<Sampled4Spectrum>();
        for (int i = 0; i < 4; ++i) {
            sa->v[i] = x[i];
            ss->v[i] = x[4 + i];
            sa->l[i] = ss->l[i] = lam[i];
        }
        HomogeneousMedium m(sa, ss, 1.f, 0.f);
        Ray ray(Vec3f(0, 0, 0), Vec3f(0, 0, 1));
        SampledSpectrum T = m.Transmittance(ray, x[8], swl);
        auto ds = m.SampleDistanceHero(ray, x[8], x[9], swl);
        for (int i = 0; i < 4; ++i) y[i] = T[i];
        y[4] = ds.scattered ? 1.f : 0.f;
        y[5] = ds.t;
        for (int i = 0; i < 4; ++i) {
            y[6 + i] = ds.weight[i];
            y[10 + i] = ds.pdfRatio[i];
        }
    }
    if (lambda4)
        for (int i = 0; i < 4; ++i) const_cast<float *>(lambda4)[i] = lam[i];
}

// ---------------------------------------------------------------------------------------------
// Spectra

API void prref_sample_visible(int64_t n, const float *u, float *lambda, float *pdf) {
    for (int64_t j = 0; j < n; ++j) {
        SampledWavelengths w = SampledWavelengths::SampleVisible(u[j]);
        SampledSpectrum p = w.PDF();
        for (int i = 0; i < 4; ++i) {
            lambda[4 * j + i] = w[i];
            pdf[4 * j + i] = p[i];
        }
    }
}

API void prref_cie(int64_t n, const float *lambda, float *xyz) {
    for (int64_t j = 0; j < n; ++j) {
        xyz[3 * j] = CIE_X(lambda[j]);
        xyz[3 * j + 1] = CIE_Y(lambda[j]);
        xyz[3 * j + 2] = CIE_Z(lambda[j]);
    }
}

API float prref_cie_y_integral() { return CIE_Y_Integral(); }

// Evaluates a spectrum at n wavelengths. kind: 0 RGB albedo (a, b, c = r, g, b), 1 RGB unbounded,
// 2 RGB illuminant, 3 blackbody normalised to Y (a = kelvin), 4 named IOR (name), 5 named metal
// eta (name), 6 named metal k (name).
API int prref_spectrum(int kind, float a, float b, float c, const char *name, int64_t n, const float *lambda,
                       float *out) {
    SpectrumPtr s;
    switch (kind) {
    case 0: s = std::make_shared<RGBAlbedoSpectrum>(RGB(a, b, c)); break;
    case 1: s = std::make_shared<RGBUnboundedSpectrum>(RGB(a, b, c)); break;
    case 2: s = std::make_shared<RGBIlluminantSpectrum>(RGB(a, b, c)); break;
    case 3: {
        SpectrumPtr bb = std::make_shared<BlackbodySpectrum>(a);
        float y = SpectrumToY(*bb);
        s = std::make_shared<ScaledSpectrum>(1 / y, bb);
        break;
    }
    case 4: s = GetNamedIOR(name ? name : ""); break;
    case 5:
    case 6: {
        SpectrumPtr e, k;
        if (GetNamedMetal(name ? name : "", &e, &k)) s = kind == 5 ? e : k;
        break;
    }
    default: break;
    }
    if (!s) return 1;
    for (int64_t j = 0; j < n; ++j) out[j] = (*s)(lambda[j]);
    return 0;
}

// ---------------------------------------------------------------------------------------------
// Scenes: load with the reference loader, export for the GPU module, render with PathIntegrator

namespace {

struct SceneHandle {
    std::unique_ptr<Scene> scene;
    // Flattened v4 scene (gpu_path.cpp:284-456 restated).
    std::vector<prgpu::Spectrum> spectra;
    std::vector<prgpu::Material> materials;
    std::vector<prgpu::Primitive> prims;
    std::vector<prgpu::Light> lights;
    std::vector<prgpu::Medium> media;
    std::vector<prgpu::BVHNode> nodes;
    std::vector<int32_t> order;
    std::vector<float> sheen;
    std::vector<float> cie;
    prgpu::SceneDesc sd{};
    std::string warnings;
    std::map<const Spectrum *, int> specCache;
    std::map<const Material *, int> matCache;
    std::map<const pr::Medium *, int> medCache;
    // Heterogeneous media, in first-use order: exported as indices mediumCount + k (the layout of
    // the GPU module's grid-media extension); their parameters come from the scene file.
    std::vector<const pr::Medium *> grids;
    // Lights outside the v4 table, in scene order: type 2 image environment, 3 sun, 4 spot,
    // 5 distant, 6 goniometric; their light-sampler pmfs (renormalised with the exported lights').
    std::vector<std::pair<int, float>> infinite;
    int interfaceMat = -1;

    int Spec(const Spectrum &s) {
        prgpu::Spectrum t;
        for (int i = 0; i < prgpu::kSpectrumSamples; ++i) t.v[i] = s(prgpu::kSpectrumMin + prgpu::kSpectrumStep * i);
        spectra.push_back(t);
        return int(spectra.size() - 1);
    }
    int Spec(const SpectrumPtr &s) {
        auto it = specCache.find(s.get());
        if (it != specCache.end()) return it->second;
        int id = Spec(*s);
        specCache[s.get()] = id;
        return id;
    }
    void Warn(const std::string &w) {
        if (warnings.find(w) == std::string::npos) warnings += w + "; ";
    }
    int SpecTex(const SpectrumTexturePtr &t, int *second, float *scale) {
        *second = -1;
        *scale = 0;
        if (auto *c = dynamic_cast<const ConstantSpectrumTexture *>(t.get())) return Spec(c->GetSpectrum());
        if (auto *ch = dynamic_cast<const CheckerSpectrumTexture *>(t.get())) {
            int d;
            float s2;
            int a = SpecTex(ch->A(), &d, &s2), b = SpecTex(ch->B(), &d, &s2);
            *second = b;
            *scale = ch->Mapping().scale.x;
            return a;
        }
        Warn("textures approximated by their average colour");
        RGB avg = t->AverageRGB();
        RGBAlbedoSpectrum s(RGB(Clamp(avg.r, 0.f, 1.f), Clamp(avg.g, 0.f, 1.f), Clamp(avg.b, 0.f, 1.f)));
        return Spec(s);
    }
    float FloatTex(const FloatTexturePtr &t, float def) {
        if (!t) return def;
        if (auto *c = dynamic_cast<const ConstantFloatTexture *>(t.get())) return c->Value();
        Warn("roughness textures approximated by a constant");
        return def;
    }
    void Conductor(const ConductorParams &p, prgpu::Material *m) {
        m->type = prgpu::MatConductor;
        float ur = FloatTex(p.uRoughness, 0.f), vr = p.vRoughness ? FloatTex(p.vRoughness, ur) : ur;
        m->alphaX = TrowbridgeReitzDistribution::RoughnessToAlpha(ur);
        m->alphaY = TrowbridgeReitzDistribution::RoughnessToAlpha(vr);
        if (p.eta && p.k) {
            int d;
            float s;
            m->eta = SpecTex(p.eta, &d, &s);
            m->k = SpecTex(p.k, &d, &s);
        } else {
            m->albedo = SpecTex(p.reflectance, &m->albedoB, &m->checkerScale);
        }
    }
    // Coat parameters of CoatedDiffuse / CoatedConductor materials (material.h:129-136).
    void Coat(const CoatParams &c, prgpu::Material *m) {
        m->coatEta = Spec(c.eta);
        m->coatDispersive = c.eta->IsConstant() ? 0 : 1;
        m->coatAlpha = TrowbridgeReitzDistribution::RoughnessToAlpha(FloatTex(c.roughness, 0.f));
        m->thickness = FloatTex(c.thickness, 0.01f);
        m->coatAlbedo = -1;
        if (c.albedo) {
            int d;
            float sc;
            m->coatAlbedo = SpecTex(c.albedo, &d, &sc);
        }
        m->coatG = c.g;
        m->coatMaxDepth = c.maxDepth;
        m->coatSamples = c.nSamples;
    }
    int MediumIndex(const pr::Medium *md) {
        if (!md) return -1;
        auto it = medCache.find(md);
        if (it != medCache.end()) return it->second;
        int id = -1;
        if (auto *h = dynamic_cast<const HomogeneousMedium *>(md)) {
            prgpu::Medium g{};
            g.sigmaA = Spec(h->SigmaAPtr());
            g.sigmaS = Spec(h->SigmaSPtr());
            g.scale = h->Scale();
            g.g = h->G();
            media.push_back(g);
            id = int(media.size() - 1);
        } else {
            // Placeholder -2 - k, resolved to mediumCount + k once every homogeneous medium is known.
            grids.push_back(md);
            id = -2 - int(grids.size() - 1);
        }
        medCache[md] = id;
        return id;
    }
    int InterfaceMat() {
        if (interfaceMat < 0) {
            prgpu::Material m{};
            m.albedo = m.albedoB = m.eta = m.k = -1;
            m.coatEta = m.coatAlbedo = m.sheenColor = -1;
            m.type = prgpu::MatInterface;
            materials.push_back(m);
            interfaceMat = int(materials.size() - 1);
        }
        return interfaceMat;
    }
    int Mat(const Material *mat) {
        auto it = matCache.find(mat);
        if (it != matCache.end()) return it->second;
        prgpu::Material m{};
        m.albedo = m.albedoB = m.eta = m.k = -1;
        m.coatEta = m.coatAlbedo = m.sheenColor = -1;
        if (!mat) {
            m.type = prgpu::MatBlack;
        } else if (auto *d = dynamic_cast<const DiffuseMaterial *>(mat)) {
            m.type = prgpu::MatDiffuse;
            m.albedo = SpecTex(d->Reflectance(), &m.albedoB, &m.checkerScale);
        } else if (auto *c = dynamic_cast<const ConductorMaterial *>(mat)) {
            Conductor(c->Params(), &m);
        } else if (auto *g = dynamic_cast<const DielectricMaterial *>(mat)) {
            m.type = prgpu::MatDielectric;
            m.eta = Spec(g->Eta());
            m.dispersive = g->IsDispersive() ? 1 : 0;
            m.thin = g->Thin() ? 1 : 0;
            float ur = FloatTex(g->URoughness(), 0.f), vr = g->VRoughness() ? FloatTex(g->VRoughness(), ur) : ur;
            m.alphaX = TrowbridgeReitzDistribution::RoughnessToAlpha(ur);
            m.alphaY = TrowbridgeReitzDistribution::RoughnessToAlpha(vr);
        } else if (auto *cd = dynamic_cast<const CoatedDiffuseMaterial *>(mat)) {
            m.albedo = SpecTex(cd->Reflectance(), &m.albedoB, &m.checkerScale);
            Coat(cd->Coat(), &m);
            m.type = prgpu::MatCoatedDiffuse;
        } else if (auto *cc = dynamic_cast<const CoatedConductorMaterial *>(mat)) {
            Conductor(cc->Conductor(), &m);
            Coat(cc->Coat(), &m);
            m.type = prgpu::MatCoatedConductor;
        } else {
            Warn("unsupported material exported as grey diffuse");
            m.type = prgpu::MatDiffuse;
            m.albedo = Spec(ConstantSpectrum(0.5f));
        }
        if (mat && mat->HasSheen() && mat->Sheen().color) {
            int d;
            float sc;
            m.sheenColor = SpecTex(mat->Sheen().color, &d, &sc);
            m.sheenRoughness = FloatTex(mat->Sheen().roughness, 0.3f);
            m.sheenWeight = mat->Sheen().weight;
        }
        materials.push_back(m);
        int id = int(materials.size() - 1);
        matCache[mat] = id;
        return id;
    }
};

} // namespace

API void *prref_scene_load(const char *path, int width, int height, char *err, int errLen) {
    std::string e;
    LoadOptions opts;
    if (width > 0) opts.width = width;
    if (height > 0) opts.height = height;
    auto scene = LoadScene(path, opts, &e);
    if (!scene) {
        SetErr(err, errLen, e);
        return nullptr;
    }
    auto *h = new SceneHandle;
    h->scene = std::move(scene);
    return h;
}

API void prref_scene_free(void *h) { delete static_cast<SceneHandle *>(h); }

API int64_t prref_scene_prim_count(void *h) { return int64_t(static_cast<SceneHandle *>(h)->scene->primitives.size()); }
API int prref_scene_width(void *h) { return static_cast<SceneHandle *>(h)->scene->settings.film.width; }
API int prref_scene_height(void *h) { return static_cast<SceneHandle *>(h)->scene->settings.film.height; }

// Flattens the loaded scene into the v4 POD layout and returns a pointer to a SceneDesc whose
// arrays live in the handle (valid until prref_scene_free). Returns nullptr on failure.
API const prgpu::SceneDesc *prref_scene_export(void *hp, char *err, int errLen) {
    auto *h = static_cast<SceneHandle *>(hp);
    const Scene &scene = *h->scene;
    auto *camera = dynamic_cast<const PerspectiveCamera *>(scene.camera.get());
    if (!camera) {
        SetErr(err, errLen, "only perspective / thin-lens cameras export");
        return nullptr;
    }
    h->prims.clear();
    for (size_t i = 0; i < scene.primitives.size(); ++i) {
        const Primitive &p = scene.primitives[i];
        prgpu::Primitive g{};
        g.light = -1;
        g.mediumInside = h->MediumIndex(p.mediumInterface.inside);
        g.mediumOutside = h->MediumIndex(p.mediumInterface.outside);
        if (auto *sp = dynamic_cast<const Sphere *>(p.shape)) {
            g.type = prgpu::PrimSphere;
            g.p0 = {sp->Center().x, sp->Center().y, sp->Center().z};
            g.r = sp->Radius();
            g.flip = sp->Flip() ? 1 : 0;
        } else if (auto *tr = dynamic_cast<const Triangle *>(p.shape)) {
            const TriangleMesh &m = tr->Mesh();
            const int *vi = &m.indices[3 * size_t(tr->Index())];
            auto F3 = [](const Vec3f &v) { return prgpu::Float3{v.x, v.y, v.z}; };
            g.type = prgpu::PrimTriangle;
            g.p0 = F3(m.p[vi[0]]);
            g.p1 = F3(m.p[vi[1]]);
            g.p2 = F3(m.p[vi[2]]);
            if (!m.n.empty()) {
                g.n0 = F3(m.n[vi[0]]);
                g.n1 = F3(m.n[vi[1]]);
                g.n2 = F3(m.n[vi[2]]);
            }
            if (!m.uv.empty()) {
                g.u0 = m.uv[vi[0]].x; g.v0 = m.uv[vi[0]].y;
                g.u1 = m.uv[vi[1]].x; g.v1 = m.uv[vi[1]].y;
                g.u2 = m.uv[vi[2]].x; g.v2 = m.uv[vi[2]].y;
            } else {
                g.u0 = 0; g.v0 = 0; g.u1 = 1; g.v1 = 0; g.u2 = 1; g.v2 = 1;
            }
        } else {
            SetErr(err, errLen, "unsupported shape");
            return nullptr;
        }
        g.material = p.IsInterface() ? h->InterfaceMat() : h->Mat(p.material);
        h->prims.push_back(g);
    }
    const int cameraMedium = h->MediumIndex(scene.camera->medium);
    float envPmf = 0, pmfSum = 0, envScale = 0;
    int envSpectrum = -1;
    for (const auto &lp : scene.lights) {
        const Light *l = lp.get();
        float pmf = scene.lightSampler.PMF(l);
        if (auto *al = dynamic_cast<const DiffuseAreaLight *>(l)) {
            int primIndex = -1;
            for (size_t i = 0; i < scene.primitives.size(); ++i)
                if (scene.primitives[i].areaLight == l) {
                    primIndex = int(i);
                    break;
                }
            if (primIndex < 0) continue;
            prgpu::Light g{};
            g.type = prgpu::LightArea;
            g.primitive = primIndex;
            g.spectrum = h->Spec(al->Emission());
            g.scale = al->Scale();
            g.twoSided = al->TwoSided() ? 1 : 0;
            g.cosPower = al->CosPower();
            g.area = al->GetShape()->Area();
            g.pmf = pmf;
            h->prims[size_t(primIndex)].light = int(h->lights.size());
            h->lights.push_back(g);
            pmfSum += pmf;
        } else if (auto *pl = dynamic_cast<const PointLight *>(l)) {
            prgpu::Light g{};
            g.type = prgpu::LightPoint;
            g.primitive = -1;
            g.spectrum = h->Spec(pl->Intensity());
            g.scale = pl->Scale();
            g.position = {pl->Position().x, pl->Position().y, pl->Position().z};
            g.pmf = pmf;
            h->lights.push_back(g);
            pmfSum += pmf;
        } else if (auto *env = dynamic_cast<const EnvironmentLight *>(l); env && env->ConstantRadiance()) {
            envSpectrum = h->Spec(env->ConstantRadiance());
            envScale = env->Scale();
            envPmf = pmf;
            pmfSum += pmf;
        } else if (dynamic_cast<const EnvironmentLight *>(l)) {
            h->infinite.push_back({2, pmf});
            pmfSum += pmf;
        } else if (dynamic_cast<const SunLight *>(l)) {
            h->infinite.push_back({3, pmf});
            pmfSum += pmf;
        } else if (dynamic_cast<const SpotLight *>(l)) {
            h->infinite.push_back({4, pmf});
            pmfSum += pmf;
        } else if (dynamic_cast<const DistantLight *>(l)) {
            h->infinite.push_back({5, pmf});
            pmfSum += pmf;
        } else if (dynamic_cast<const GoniometricLight *>(l)) {
            h->infinite.push_back({6, pmf});
            pmfSum += pmf;
        } else {
            h->Warn("light type not exported");
        }
    }
    if (pmfSum > 0) {
        for (auto &l : h->lights) l.pmf /= pmfSum;
        envPmf /= pmfSum;
        for (auto &i : h->infinite) i.second /= pmfSum;
    }
    const BVH &bvh = scene.GetBVH();
    h->nodes.clear();
    for (const auto &n : bvh.Nodes()) {
        prgpu::BVHNode g{};
        g.bmin = {n.bounds.pMin.x, n.bounds.pMin.y, n.bounds.pMin.z};
        g.bmax = {n.bounds.pMax.x, n.bounds.pMax.y, n.bounds.pMax.z};
        g.offset = n.offset;
        g.nPrims = n.nPrims;
        g.axis = n.axis;
        h->nodes.push_back(g);
    }
    h->order = bvh.Order();
    prgpu::SceneDesc &sd = h->sd;
    sd = prgpu::SceneDesc{};
    sd.apiVersion = prgpu::kApiVersion;
    sd.nodes = h->nodes.data();
    sd.nodeCount = int(h->nodes.size());
    sd.primOrder = h->order.data();
    sd.prims = h->prims.data();
    sd.primCount = int(h->prims.size());
    sd.materials = h->materials.data();
    sd.materialCount = int(h->materials.size());
    sd.lights = h->lights.data();
    sd.lightCount = int(h->lights.size());
    sd.spectra = h->spectra.data();
    sd.spectrumCount = int(h->spectra.size());
    sd.media = h->media.data();
    sd.mediumCount = int(h->media.size());
    auto resolve = [&](int32_t id) { return id <= -2 ? sd.mediumCount + (-2 - id) : id; };
    for (prgpu::Primitive &g : h->prims) {
        g.mediumInside = resolve(g.mediumInside);
        g.mediumOutside = resolve(g.mediumOutside);
    }
    sd.cameraMedium = resolve(cameraMedium);
    sd.envSpectrum = envSpectrum;
    sd.envScale = envScale;
    sd.envPmf = envPmf;
    sd.worldCenter = {scene.worldCenter.x, scene.worldCenter.y, scene.worldCenter.z};
    sd.worldRadius = scene.worldRadius;
    const Mat4 &m = camera->CameraToWorld().Matrix();
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) sd.camera.cameraToWorld[r * 4 + c] = m.m[r][c];
    const FilmSettings &fs = scene.settings.film;
    sd.camera.tanHalfFov = camera->TanHalfFov();
    sd.camera.aspect = float(fs.width) / fs.height;
    sd.camera.lensRadius = camera->LensRadius();
    sd.camera.focalDistance = camera->FocalDistance();
    sd.camera.width = fs.width;
    sd.camera.height = fs.height;
    sd.camera.margin = 0;
    sd.cieYIntegral = CIE_Y_Integral();
    h->sheen.assign(size_t(prgpu::kSheenAlpha) * prgpu::kSheenMu, 0.f);
    for (int ia = 0; ia < prgpu::kSheenAlpha; ++ia)
        for (int im = 0; im < prgpu::kSheenMu; ++im)
            h->sheen[size_t(ia) * prgpu::kSheenMu + im] =
                SheenBxDF::Albedo(float(im) / (prgpu::kSheenMu - 1), 0.05f + 0.95f * float(ia) / (prgpu::kSheenAlpha - 1));
    sd.sheenAlbedo = h->sheen.data();
    h->cie.resize(3 * prgpu::kSpectrumSamples);
    for (int i = 0; i < prgpu::kSpectrumSamples; ++i) {
        float l = prgpu::kSpectrumMin + prgpu::kSpectrumStep * i;
        h->cie[i] = CIE_X(l);
        h->cie[prgpu::kSpectrumSamples + i] = CIE_Y(l);
        h->cie[2 * prgpu::kSpectrumSamples + i] = CIE_Z(l);
    }
    sd.cie = h->cie.data();
    Filter filter(fs.filter);
    sd.filter.type = filter.Type() == FilterType::Gaussian        ? prgpu::FilterGaussian
                     : filter.Type() == FilterType::BlackmanHarris ? prgpu::FilterBlackmanHarris
                                                                   : prgpu::FilterBox;
    sd.filter.radius = filter.Radius();
    sd.filter.sigma = filter.Sigma();
    sd.filter.norm = filter.Norm();
    {
        double sum = 0, peak = 0, bins[prgpu::kFilterBins];
        for (int i = 0; i < prgpu::kFilterBins; ++i) {
            float x = -filter.Radius() + (i + 0.5f) * (2 * filter.Radius() / prgpu::kFilterBins);
            bins[i] = std::abs(filter.Eval1D(x));
            peak = std::max(peak, bins[i]);
        }
        for (double &b : bins) b += 1e-3 * peak;
        for (double b : bins) sum += b;
        double acc = 0;
        sd.filter.cdf[0] = 0;
        for (int i = 0; i < prgpu::kFilterBins; ++i) {
            acc += bins[i] / sum;
            sd.filter.cdf[i + 1] = float(acc);
        }
        sd.filter.cdf[prgpu::kFilterBins] = 1;
    }
    if (!h->warnings.empty()) SetErr(err, errLen, h->warnings);
    return &h->sd;
}

// Renders the scene with the reference CPU path tracer (PathIntegrator, box or scene filter) and
// writes per-pixel XYZ SUMS over the spp samples (unscaled) into out[3*w*h]. lightBVH selects the
// light-BVH sampler (1) or the power sampler (0). Returns elapsed seconds, or -1 on failure.
API double prref_render(void *hp, int spp, uint64_t seed, int maxDepth, int lightBVH, float *out, char *err, int errLen) {
    auto *h = static_cast<SceneHandle *>(hp);
    const Scene &scene = *h->scene;
    IntegratorSettings is = scene.settings.integrator;
    is.type = IntegratorType::Path;
    is.device = -1;
    is.spp = spp;
    is.maxDepth = maxDepth;
    is.timeLimit = 0;
    is.lightBVH = lightBVH != 0;
    auto integrator = CreateIntegrator(is, seed);
    Film film(scene.settings.film);
    RenderControl control;
    control.Start();
    double scale = 0;
    std::string e;
    auto t0 = std::chrono::steady_clock::now();
    if (!integrator->Render(scene, film, control, &scale, &e)) {
        SetErr(err, errLen, e);
        return -1;
    }
    double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const int w = film.Width(), hh = film.Height();
    for (int y = 0; y < hh; ++y)
        for (int x = 0; x < w; ++x) {
            XYZ v = film.PixelXYZ(x, y);
            size_t i = 3 * (size_t(y) * w + x);
            out[i] = v.x;
            out[i + 1] = v.y;
            out[i + 2] = v.z;
        }
    return dt;
}

// Light-BVH selection at shading points: in (per item, 7 floats) p[3], n[3], u. out (per item,
// 2 floats): chosen light index in scene.lights (-1 none), pmf. pmfOut (per item x lightCount):
// BVHLightSampler::PMF for every light at that point (nullptr to skip).
API void prref_light_bvh_sample(void *hp, int64_t n, const float *in, float *out, float *pmfOut) {
    auto *h = static_cast<SceneHandle *>(hp);
    const Scene &scene = *h->scene;
    std::map<const Light *, int> index;
    for (size_t i = 0; i < scene.lights.size(); ++i) index[scene.lights[i].get()] = int(i);
    for (int64_t j = 0; j < n; ++j) {
        const float *x = in + 7 * j;
        Vec3f p(x[0], x[1], x[2]), nn(x[3], x[4], x[5]);
        float pmf = 0;
        const Light *l = scene.lightBVH.Sample(p, nn, x[6], &pmf);
        out[2 * j] = l ? float(index[l]) : -1.f;
        out[2 * j + 1] = l ? pmf : 0.f;
        if (pmfOut)
            for (size_t i = 0; i < scene.lights.size(); ++i)
                pmfOut[j * int64_t(scene.lights.size()) + int64_t(i)] = scene.lightBVH.PMF(p, nn, scene.lights[i].get());
    }
}

API int prref_scene_light_count(void *hp) { return int(static_cast<SceneHandle *>(hp)->scene->lights.size()); }

// Heterogeneous media of the last export (index mediumCount + k): their names in the scene file and
// the density-field bounds in medium space after the loader fitted them (scene_loader.cpp:1302-1308).
// Infinite lights of the last export other than the constant environment (the GPU module's
// SceneExt::envMap / sun): count, then per light its type (2 image environment, 3 sun) and pmf.
API int prref_scene_infinite(void *hp, int max, int *types, float *pmfs) {
    auto *h = static_cast<SceneHandle *>(hp);
    int n = int(h->infinite.size());
    for (int i = 0; i < std::min(n, max); ++i) {
        types[i] = h->infinite[size_t(i)].first;
        pmfs[i] = h->infinite[size_t(i)].second;
    }
    return n;
}

// The reference's RGB uplift of unbounded RGB values (RGBUnboundedSample, rgb2spec.cpp:328-336) as
// sigmoid-polynomial coefficients: out 4 floats per colour (c0, c1, c2, scale), reconstructed from
// the polynomial's values at 400, 550 and 700 nm (its coefficients are not exposed).
API void prref_rgb_uplift(int64_t n, const float *rgb, float *out) {
    const RGBToSpectrumTable &table = RGBToSpectrumTable::Get();
    for (int64_t i = 0; i < n; ++i) {
        RGB c(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]);
        float m = std::max(0.f, c.Max());
        float *o = out + 4 * i;
        if (m == 0.f) {
            o[0] = o[1] = o[2] = 0.f;
            o[3] = 0.f;
            continue;
        }
        float scale = 2 * m;
        RGBSigmoidPolynomial rsp = table(c * (1 / scale));
        const double L[3] = {400.0, 550.0, 700.0};
        double x[3];
        for (int k = 0; k < 3; ++k) {
            double y = 2.0 * double(rsp(float(L[k]))) - 1.0;
            y = std::max(-0.999999, std::min(0.999999, y));
            x[k] = y / std::sqrt(1.0 - y * y);
        }
        // Quadratic through (L_k, x_k): c0 l^2 + c1 l + c2.
        double d01 = (x[1] - x[0]) / (L[1] - L[0]), d12 = (x[2] - x[1]) / (L[2] - L[1]);
        double c0 = (d12 - d01) / (L[2] - L[0]);
        double c1 = d01 - c0 * (L[0] + L[1]);
        double c2 = x[0] - c0 * L[0] * L[0] - c1 * L[0];
        o[0] = float(c0);
        o[1] = float(c1);
        o[2] = float(c2);
        o[3] = scale;
    }
}

// MakePreethamSky (sky.cpp:146-205): linear RGB, width x height x 3.
API void prref_preetham_sky(const float *sunDir, float turbidity, float groundAlbedo, int width, int height, float *rgb) {
    auto img = MakePreethamSky(Normalize(Vec3f(sunDir[0], sunDir[1], sunDir[2])), turbidity, groundAlbedo, width, height);
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            RGB c = img->Get(x, y);
            float *o = rgb + 3 * (size_t(y) * width + x);
            o[0] = c.r;
            o[1] = c.g;
            o[2] = c.b;
        }
}

// MakeSunRadiance (sky.cpp:207-233) at n wavelengths.
API void prref_sun_radiance(const float *sunDir, float turbidity, float radiusDeg, int64_t n, const float *lambda,
                            float *out) {
    auto s = MakeSunRadiance(Normalize(Vec3f(sunDir[0], sunDir[1], sunDir[2])), turbidity, radiusDeg);
    for (int64_t i = 0; i < n; ++i) out[i] = (*s)(lambda[i]);
}

API int prref_scene_grid_count(void *hp) { return int(static_cast<SceneHandle *>(hp)->grids.size()); }

API int prref_scene_grid_info(void *hp, int k, char *name, int nameLen, float *bounds6) {
    auto *h = static_cast<SceneHandle *>(hp);
    if (k < 0 || k >= int(h->grids.size())) return -1;
    auto *gm = dynamic_cast<const GridMedium *>(h->grids[size_t(k)]);
    if (!gm) return -1;
    std::snprintf(name, size_t(nameLen), "%s", gm->name.c_str());
    const Bounds3f &b = const_cast<GridMedium *>(gm)->Field().bounds;
    for (int a = 0; a < 3; ++a) {
        bounds6[a] = b.pMin[a];
        bounds6[3 + a] = b.pMax[a];
    }
    return 0;
}

// pr::RenderAOV on the loaded scene (type: 0 albedo, 1 normal, 2 depth, 3 position) into
// out[width * height * 3]; and the two colour matrices its albedo uses (white adaptation of the
// spectral D65 white, then XYZ -> linear sRGB; color.cpp:92-99), row-major.
API void prref_render_aov(void *hp, int type, int spp, uint64_t seed, int throughSpecular, float *out) {
    auto *h = static_cast<SceneHandle *>(hp);
    Image img = RenderAOV(*h->scene, AOVType(type), spp, seed, throughSpecular != 0);
    for (int y = 0; y < img.Height(); ++y)
        for (int x = 0; x < img.Width(); ++x) {
            RGB c = img.Get(x, y);
            float *o = out + 3 * (size_t(y) * img.Width() + x);
            o[0] = c.r;
            o[1] = c.g;
            o[2] = c.b;
        }
}

API void prref_aov_matrices(float *adapt9, float *toRGB9) {
    const Mat3 &a = SpectralWhiteAdaptation(), &m = XYZToRGBMatrix(ColorSpaceId::sRGB);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            adapt9[3 * i + j] = a.m[i][j];
            toRGB9[3 * i + j] = m.m[i][j];
        }
}

// ---------------------------------------------------------------------------------------------
// NanoVDB fixtures and field samples: a fog sphere written with NanoVDB's own tools (as the
// reference's tests/test_media.cpp:134-143 makes one), and the density of a loaded scene's grid
// medium k at medium-space points (pr::DensityField::Density, media/nanovdb_field.cpp:27-39 for a
// NanoVDB field).
#include <nanovdb/tools/CreatePrimitives.h>
#include <fstream>

API int prref_write_fog_sphere(const char *path, double radius, double voxelSize, double halfWidth) {
    auto handle = nanovdb::tools::createFogVolumeSphere<float>(radius, nanovdb::Vec3d(0.0), voxelSize, halfWidth,
                                                               nanovdb::Vec3d(0.0), "density");
    std::ofstream os(path, std::ios::binary);
    if (!os) return 1;
    nanovdb::io::writeUncompressedGrid(os, handle.gridData());
    return os.good() ? 0 : 1;
}

API int prref_scene_grid_density(void *hp, int k, int64_t n, const float *pts, float *out) {
    auto *h = static_cast<SceneHandle *>(hp);
    if (k < 0 || k >= int(h->grids.size())) return -1;
    auto *gm = dynamic_cast<const GridMedium *>(h->grids[size_t(k)]);
    if (!gm) return -1;
    const DensityField &f = const_cast<GridMedium *>(gm)->Field();
    for (int64_t i = 0; i < n; ++i) out[i] = f.Density(Vec3f(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]));
    return 0;
}
