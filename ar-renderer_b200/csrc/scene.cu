// Scene upload: validation of the caller's SceneDesc (every index a kernel will follow is range-
// checked on the host, so malformed input is an error return, never a device fault), conversion
// of the BVH, and a content-keyed cache so progressive batches upload once. The reference keys
// its cache on the primitive pointer and counts only (src/gpu/prender_gpu.cpp:1653-1670) and so
// misses an edited scene behind the same pointer; here the key also hashes the small tables in
// full and a strided sample of the large ones.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "scene.cuh"

namespace prb {

namespace {

uint64_t fnv(uint64_t h, const void *p, size_t n) {
    const unsigned char *b = static_cast<const unsigned char *>(p);
    for (size_t i = 0; i < n; ++i) {
        h ^= b[i];
        h *= 0x100000001b3ull;
    }
    return h;
}
template <typename T> uint64_t fnv_v(uint64_t h, const T &v) { return fnv(h, &v, sizeof(T)); }

// Hash of up to `samples` evenly strided elements plus the first and last.
uint64_t sample_hash(uint64_t h, const void *base, size_t count, size_t elem, size_t samples) {
    if (!base || count == 0) return fnv_v(h, count);
    const unsigned char *b = static_cast<const unsigned char *>(base);
    size_t step = std::max<size_t>(1, count / samples);
    for (size_t i = 0; i < count; i += step) h = fnv(h, b + i * elem, elem);
    return fnv(h, b + (count - 1) * elem, elem);
}

uint64_t scene_key(const prgpu::SceneDesc *sd, const prgpu::SceneExt *ext) {
    uint64_t h = 0xcbf29ce484222325ull;
    h = fnv_v(h, sd->prims);
    h = fnv_v(h, sd->nodes);
    h = fnv_v(h, sd->primCount);
    h = fnv_v(h, sd->nodeCount);
    h = sample_hash(h, sd->prims, size_t(sd->primCount), sizeof(prgpu::Primitive), 4096);
    h = sample_hash(h, sd->nodes, size_t(sd->nodeCount), sizeof(prgpu::BVHNode), 4096);
    h = sample_hash(h, sd->primOrder, size_t(sd->primCount), sizeof(int32_t), 4096);
    if (sd->materials) h = fnv(h, sd->materials, size_t(sd->materialCount) * sizeof(prgpu::Material));
    if (sd->lights) h = fnv(h, sd->lights, size_t(sd->lightCount) * sizeof(prgpu::Light));
    if (sd->spectra) h = fnv(h, sd->spectra, size_t(sd->spectrumCount) * sizeof(prgpu::Spectrum));
    if (sd->media) h = fnv(h, sd->media, size_t(sd->mediumCount) * sizeof(prgpu::Medium));
    h = fnv(h, sd->filter.cdf, sizeof(sd->filter.cdf));
    if (ext && ext->lightBVH && ext->lightBVHNodeCount > 0)
        h = fnv(h, ext->lightBVH, size_t(ext->lightBVHNodeCount) * sizeof(prgpu::LightBVHNode));
    if (ext && ext->envMap) {
        h = fnv_v(h, *ext->envMap);
        h = sample_hash(h, ext->envMap->texels, size_t(std::max(0, ext->envMap->width)) * size_t(std::max(0, ext->envMap->height)),
                        4 * sizeof(float), 65536);
    }
    if (ext && ext->sun) h = fnv_v(h, *ext->sun);
    if (ext && ext->textureNodes && ext->textureNodeCount > 0)
        h = fnv(h, ext->textureNodes, size_t(ext->textureNodeCount) * sizeof(prgpu::TextureNode));
    if (ext && ((ext->textures && ext->textureCount > 0) || (ext->textureNodes && ext->textureNodeCount > 0))) {
        for (int32_t k = 0; ext->textures && k < ext->textureCount; ++k) {
            const prgpu::ImageTextureDesc &t = ext->textures[k];
            h = fnv_v(h, t);
            h = sample_hash(h, t.rgb, size_t(std::max(0, t.width)) * size_t(std::max(0, t.height)), 3 * sizeof(float), 65536);
        }
        if (ext->materialTextures && ext->materialTextureCount > 0)
            h = fnv(h, ext->materialTextures, size_t(ext->materialTextureCount) * sizeof(prgpu::MaterialTextures));
        h = fnv_v(h, ext->rgbToSpectrum);
    }
    if (ext && ext->deltaLights && ext->deltaLightCount > 0)
        for (int32_t k = 0; k < ext->deltaLightCount; ++k) {
            const prgpu::DeltaLightDesc &l = ext->deltaLights[k];
            h = fnv_v(h, l);
            if (l.type == prgpu::DeltaGoniometric && l.profile && l.nV > 0 && l.nH > 0)
                h = fnv(h, l.profile, (size_t(l.nV) + size_t(l.nH) + size_t(l.nV) * size_t(l.nH)) * sizeof(float));
        }
    if (ext && ext->gridMedia && ext->gridMediumCount > 0)
        for (int32_t k = 0; k < ext->gridMediumCount; ++k) {
            const prgpu::GridMediumDesc &g = ext->gridMedia[k];
            h = fnv_v(h, g);
            if (g.field != prgpu::GridNoise)
                h = sample_hash(h, g.density, size_t(g.nx) * size_t(g.ny) * size_t(g.nz), sizeof(float), 65536);
        }
    return h;
}

bool spec_ok(int32_t id, int32_t n) { return id >= -1 && id < n; }

// A texture tree rooted at `node` (-1 none): indices in range, at most 8 nodes deep (so no
// cycles), noise only as a float texture or as the blend of a mix, constants of spectrum trees
// naming a spectrum.
bool texture_tree_ok(const prgpu::SceneExt *ext, const prgpu::SceneDesc *sd, int32_t node, bool spectrum, int depth) {
    if (node == -1) return depth > 0 ? false : true;
    if (node < 0 || node >= ext->textureNodeCount || depth >= 8) return false;
    const prgpu::TextureNode &t = ext->textureNodes[node];
    switch (t.type) {
    case prgpu::TexConstant:
        return spectrum ? (t.a >= 0 && t.a < sd->spectrumCount) : std::isfinite(t.value);
    case prgpu::TexImage:
        return t.a >= 0 && t.a < ext->textureCount && t.channel >= -1 && t.channel <= 2;
    case prgpu::TexChecker:
        return std::isfinite(t.scaleU) && std::isfinite(t.scaleV) && std::isfinite(t.offsetU) &&
               std::isfinite(t.offsetV) && texture_tree_ok(ext, sd, t.a, spectrum, depth + 1) &&
               texture_tree_ok(ext, sd, t.b, spectrum, depth + 1);
    case prgpu::TexNoise:
        return !spectrum && t.octaves >= 1 && t.octaves <= 32 && std::isfinite(t.frequency) &&
               std::isfinite(t.offset[0]) && std::isfinite(t.offset[1]) && std::isfinite(t.offset[2]);
    case prgpu::TexMix:
        return t.t >= 0 && t.t < ext->textureNodeCount && ext->textureNodes[t.t].type == prgpu::TexNoise &&
               texture_tree_ok(ext, sd, t.t, false, depth + 1) && texture_tree_ok(ext, sd, t.a, spectrum, depth + 1) &&
               texture_tree_ok(ext, sd, t.b, spectrum, depth + 1);
    default: return false;
    }
}

// True when the (already validated) tree looks up an image.
bool texture_tree_has_image(const prgpu::SceneExt *ext, int32_t node, int depth) {
    if (node < 0 || depth >= 8) return false;
    const prgpu::TextureNode &t = ext->textureNodes[node];
    if (t.type == prgpu::TexImage) return true;
    if (t.type == prgpu::TexChecker || t.type == prgpu::TexMix)
        return texture_tree_has_image(ext, t.a, depth + 1) || texture_tree_has_image(ext, t.b, depth + 1);
    return false;
}

bool validate(const prgpu::SceneDesc *sd, const prgpu::SceneExt *ext, std::string *err) {
    auto fail = [&](const std::string &m) {
        *err = m;
        return false;
    };
    if (sd->primCount < 0 || sd->nodeCount < 0 || sd->materialCount < 0 || sd->lightCount < 0 ||
        sd->spectrumCount < 0 || sd->mediumCount < 0)
        return fail("negative array count");
    if ((sd->primCount > 0 && !sd->prims) || (sd->materialCount > 0 && !sd->materials) ||
        (sd->lightCount > 0 && !sd->lights) || (sd->spectrumCount > 0 && !sd->spectra) ||
        (sd->mediumCount > 0 && !sd->media))
        return fail("null scene array");
    const prgpu::Camera &c = sd->camera;
    if (c.width <= 0 || c.height <= 0 || int64_t(c.width) * c.height > (int64_t(1) << 28))
        return fail("camera resolution out of range");
    if (!std::isfinite(c.tanHalfFov) || c.tanHalfFov <= 0) return fail("bad camera field of view");
    const int32_t ns = sd->spectrumCount;
    const int32_t ng = (ext && ext->gridMediumCount > 0) ? ext->gridMediumCount : 0;
    const int32_t nm = sd->mediumCount + ng;  // homogeneous media, then grid media
    if (ng > 0 && !ext->gridMedia) return fail("null grid media");
    for (int32_t k = 0; k < ng; ++k) {
        const prgpu::GridMediumDesc &g = ext->gridMedia[k];
        if (g.field > prgpu::GridIndexed) return fail("unknown grid medium field");
        if (g.field == prgpu::GridIndexed &&
            !(g.boundsMin.x < g.boundsMax.x && g.boundsMin.y < g.boundsMax.y && g.boundsMin.z < g.boundsMax.z))
            return fail("index-space grids need non-empty bounds");
        if (g.field == prgpu::GridNoise) {
            if (g.noiseOctaves < 1 || g.noiseOctaves > 32 || !std::isfinite(g.noiseFrequency) ||
                !std::isfinite(g.noiseThreshold) || !std::isfinite(g.noiseSharpness) || !std::isfinite(g.noiseOffset[0]) ||
                !std::isfinite(g.noiseOffset[1]) || !std::isfinite(g.noiseOffset[2]))
                return fail("bad noise medium parameters");
            // Empty bounds (Bounds3f::IsEmpty, math.h:212: min > max on an axis) or a box of positive
            // extent; a degenerate box would divide the falloff by zero.
            const bool empty = g.boundsMin.x > g.boundsMax.x || g.boundsMin.y > g.boundsMax.y ||
                               g.boundsMin.z > g.boundsMax.z;
            if (!empty &&
                !(g.boundsMin.x < g.boundsMax.x && g.boundsMin.y < g.boundsMax.y && g.boundsMin.z < g.boundsMax.z))
                return fail("noise media need bounds of positive extent, or empty bounds");
        } else if (g.nx <= 0 || g.ny <= 0 || g.nz <= 0 || int64_t(g.nx) * g.ny * g.nz > (int64_t(1) << 31) || !g.density) {
            return fail("bad grid medium dimensions or data");
        }
        if (!spec_ok(g.sigmaA, ns) || !spec_ok(g.sigmaS, ns)) return fail("grid medium spectrum index out of range");
        // A noise field's bounds may be empty (min >= max on an axis): the field then has no bounds.
        if (g.field != prgpu::GridNoise &&
            !(g.boundsMin.x <= g.boundsMax.x && g.boundsMin.y <= g.boundsMax.y && g.boundsMin.z <= g.boundsMax.z))
            return fail("empty grid medium bounds");
    }
    if (!spec_ok(sd->envSpectrum, ns)) return fail("envSpectrum out of range");
    if (ext && ext->envMap) {
        const prgpu::EnvMapDesc &e = *ext->envMap;
        if (e.width <= 0 || e.height <= 0 || int64_t(e.width) * e.height > (int64_t(1) << 26) || !e.texels)
            return fail("bad environment map dimensions or data");
        if (!spec_ok(e.illuminant, ns)) return fail("environment map illuminant out of range");
        if (!(e.pmf >= 0.f && e.pmf <= 1.f) || !std::isfinite(e.scale)) return fail("bad environment map pmf or scale");
    }
    if (ext && ext->sun) {
        const prgpu::SunDesc &u = *ext->sun;
        if (u.spectrum < 0 || u.spectrum >= ns) return fail("sun spectrum index out of range");
        if (!(u.cosThetaMax > -1.f && u.cosThetaMax < 1.f) || !(u.pmf >= 0.f && u.pmf <= 1.f))
            return fail("bad sun cone or pmf");
        float l2 = u.direction.x * u.direction.x + u.direction.y * u.direction.y + u.direction.z * u.direction.z;
        if (!(l2 > 0.f) || !std::isfinite(l2)) return fail("bad sun direction");
    }
    if (ext && (ext->textureCount < 0 || ext->textureCount > 65536 || (ext->textureCount > 0 && !ext->textures) ||
                (ext->materialTextureCount != 0 && ext->materialTextureCount != sd->materialCount) ||
                (ext->materialTextureCount > 0 && !ext->materialTextures)))
        return fail("bad texture tables");
    for (int32_t k = 0; ext && k < ext->textureCount; ++k) {
        const prgpu::ImageTextureDesc &t = ext->textures[k];
        if (t.width <= 0 || t.height <= 0 || int64_t(t.width) * t.height > (int64_t(1) << 28) || !t.rgb || t.wrap > 2)
            return fail("bad image texture");
    }
    if (ext && (ext->textureNodeCount < 0 || ext->textureNodeCount > 65536 ||
                (ext->textureNodeCount > 0 && !ext->textureNodes)))
        return fail("bad texture node table");
    for (int32_t i = 0; ext && i < ext->materialTextureCount; ++i) {
        const prgpu::MaterialTextures &x = ext->materialTextures[i];
        if (!texture_tree_ok(ext, sd, x.reflectanceNode, true, 0) || !texture_tree_ok(ext, sd, x.bumpNode, false, 0) ||
            !texture_tree_ok(ext, sd, x.roughnessNodeU, false, 0) || !texture_tree_ok(ext, sd, x.roughnessNodeV, false, 0) ||
            !texture_tree_ok(ext, sd, x.coatRoughnessNode, false, 0) || !texture_tree_ok(ext, sd, x.thicknessNode, false, 0) ||
            !texture_tree_ok(ext, sd, x.coatAlbedoNode, true, 0) || !texture_tree_ok(ext, sd, x.sheenColorNode, true, 0) ||
            !texture_tree_ok(ext, sd, x.sheenRoughnessNode, false, 0) || !texture_tree_ok(ext, sd, x.etaNode, true, 0) ||
            !texture_tree_ok(ext, sd, x.kNode, true, 0) || ((x.etaNode >= 0) != (x.kNode >= 0)))
            return fail("bad texture tree (index out of range, deeper than 8 nodes, or a node of the wrong kind)");
        if (!ext->rgbToSpectrum && (texture_tree_has_image(ext, x.reflectanceNode, 0) ||
                                    texture_tree_has_image(ext, x.coatAlbedoNode, 0) ||
                                    texture_tree_has_image(ext, x.sheenColorNode, 0) ||
                                    texture_tree_has_image(ext, x.etaNode, 0) || texture_tree_has_image(ext, x.kNode, 0)))
            return fail("textured materials need the RGB -> spectrum table");
        if (!std::isfinite(x.bumpScale)) return fail("bad bump map scale");
    }
    for (int32_t i = 0; ext && i < ext->materialTextureCount; ++i) {
        const int32_t r = ext->materialTextures[i].reflectance, nmap = ext->materialTextures[i].normalMap;
        const int32_t bmap = ext->materialTextures[i].bumpMap, bch = ext->materialTextures[i].bumpChannel;
        if (r < -1 || r >= ext->textureCount || nmap < -1 || nmap >= ext->textureCount || bmap < -1 ||
            bmap >= ext->textureCount || bch < -1 || bch > 2)
            return fail("material texture index out of range");
        if (r >= 0 && !ext->rgbToSpectrum) return fail("textured materials need the RGB -> spectrum table");
        if (!std::isfinite(ext->materialTextures[i].normalStrength)) return fail("bad normal map strength");
    }
    if (ext && (ext->deltaLightCount < 0 || ext->deltaLightCount > 4096 || (ext->deltaLightCount > 0 && !ext->deltaLights)))
        return fail("bad delta light count or table");
    for (int32_t k = 0; ext && k < ext->deltaLightCount; ++k) {
        const prgpu::DeltaLightDesc &l = ext->deltaLights[k];
        if (l.type > prgpu::DeltaGoniometric) return fail("unknown delta light type");
        if (l.spectrum < 0 || l.spectrum >= ns) return fail("delta light spectrum index out of range");
        if (!(l.pmf >= 0.f && l.pmf <= 1.f) || !std::isfinite(l.scale)) return fail("bad delta light pmf or scale");
        float l2 = l.direction.x * l.direction.x + l.direction.y * l.direction.y + l.direction.z * l.direction.z;
        if (l.type != prgpu::DeltaGoniometric && !(l2 > 0.f && std::isfinite(l2))) return fail("bad delta light direction");
        if (l.type == prgpu::DeltaGoniometric &&
            (l.nV <= 0 || l.nH <= 0 || int64_t(l.nV) * l.nH > (int64_t(1) << 22) || !l.profile))
            return fail("bad goniometric profile");
    }
    if (sd->cameraMedium < -1 || sd->cameraMedium >= nm) return fail("cameraMedium out of range");
    for (int32_t i = 0; i < sd->materialCount; ++i) {
        const prgpu::Material &m = sd->materials[i];
        if (m.type > prgpu::MatCoatedConductor) return fail("unknown material type");
        if (m.type == prgpu::MatCoatedDiffuse || m.type == prgpu::MatCoatedConductor) {
            if (!spec_ok(m.coatEta, ns) || (m.coatAlbedo >= 0 && !spec_ok(m.coatAlbedo, ns)))
                return fail("coat spectrum index out of range");
            if (m.coatMaxDepth < 0 || m.coatMaxDepth > 4096 || m.coatSamples < 0 || m.coatSamples > 4096)
                return fail("coat walk depth / sample count out of range [0, 4096]");
            if (!(m.thickness >= 0.f) || !std::isfinite(m.thickness)) return fail("bad coat thickness");
        }
        if (m.sheenWeight > 0 && m.sheenColor >= 0 && !spec_ok(m.sheenColor, ns))
            return fail("sheen spectrum index out of range");
        if (!spec_ok(m.albedo, ns) || !spec_ok(m.albedoB, ns) || !spec_ok(m.eta, ns) || !spec_ok(m.k, ns))
            return fail("material spectrum index out of range");
    }
    for (int32_t i = 0; i < sd->lightCount; ++i) {
        const prgpu::Light &l = sd->lights[i];
        if (l.type > prgpu::LightPoint) return fail("unknown light type");
        if (!spec_ok(l.spectrum, ns)) return fail("light spectrum index out of range");
        if (l.type == prgpu::LightArea && (l.primitive < 0 || l.primitive >= sd->primCount))
            return fail("area light primitive out of range");
    }
    for (int32_t i = 0; i < sd->mediumCount; ++i)
        if (!spec_ok(sd->media[i].sigmaA, ns) || !spec_ok(sd->media[i].sigmaS, ns))
            return fail("medium spectrum index out of range");
    for (int32_t i = 0; i < sd->primCount; ++i) {
        const prgpu::Primitive &p = sd->prims[i];
        if (p.type > prgpu::PrimSphere) return fail("unknown primitive type");
        if (p.material < 0 || p.material >= sd->materialCount) return fail("primitive material out of range");
        if (p.light < -1 || p.light >= sd->lightCount) return fail("primitive light out of range");
        if (p.mediumInside < -1 || p.mediumInside >= nm || p.mediumOutside < -1 || p.mediumOutside >= nm)
            return fail("primitive medium out of range");
    }
    if (ext && ext->lightBVHNodeCount > 0) {
        if (!ext->lightBVH) return fail("null light BVH");
        int32_t n = ext->lightBVHNodeCount;
        for (int32_t i = 0; i < n; ++i) {
            const prgpu::LightBVHNode &b = ext->lightBVH[i];
            if (b.light >= 0) {
                if (b.light >= sd->lightCount) return fail("light BVH leaf out of range");
            } else if (b.child1 <= i + 1 || b.child1 >= n || i + 1 >= n) {
                return fail("malformed light BVH interior node");
            }
            if (b.parent >= i || b.parent < -1 || (i > 0 && b.parent < 0)) return fail("malformed light BVH parent link");
        }
    }
    return true;
}

template <typename T> void put(DevBuf &b, const T *src, size_t n, cudaStream_t s) {
    b.ensure(std::max<size_t>(1, n) * sizeof(T));
    if (n) PRB_CUDA(cudaMemcpyAsync(b.ptr, src, n * sizeof(T), cudaMemcpyHostToDevice, s));
}

// Texel radiance at wavelength l (nm): scale * S(c0 l^2 + c1 l + c2) (rgb2spec.h:13-26).
float texel_value(const float *t, float l) {
    float x = std::fma(l, std::fma(l, t[0], t[1]), t[2]);
    float s = std::isinf(x) ? (x > 0.f ? 1.f : 0.f) : 0.5f + x / (2.f * std::sqrt(1.f + x * x));
    return t[3] * s;
}

} // namespace

// The sheen lobe's directional albedo on [16 roughness] x [32 cos theta] nodes, for a host that
// passes no table: the reference's SheenBxDF::Albedo integration (bxdf.cpp:538-560) restated --
// 32 x 32 stratified cosine-weighted directions (concentric disk), f cos / pdf averaged in double.
std::vector<float> sheen_albedo_table() {
    const int nMu = prgpu::kSheenMu, nAlpha = prgpu::kSheenAlpha, nS = 32;
    std::vector<float> t(size_t(nMu) * nAlpha);
    const float pi = 3.14159265358979f;
    for (int ia = 0; ia < nAlpha; ++ia) {
        const float a = (1.f - float(ia) / (nAlpha - 1)) * 0.05f + float(ia) / (nAlpha - 1) * 1.f;
        for (int im = 0; im < nMu; ++im) {
            const float mu = std::max(1e-3f, float(im) / (nMu - 1));
            const float wo[3] = {std::sqrt(std::max(0.f, 1 - mu * mu)), 0.f, mu};
            double sum = 0;
            for (int i = 0; i < nS; ++i)
                for (int j = 0; j < nS; ++j) {
                    float ox = 2.f * ((i + 0.5f) / nS) - 1.f, oy = 2.f * ((j + 0.5f) / nS) - 1.f, x = 0.f, y = 0.f;
                    if (ox != 0.f || oy != 0.f) {
                        float r, th;
                        if (std::fabs(ox) > std::fabs(oy)) {
                            r = ox;
                            th = pi / 4 * (oy / ox);
                        } else {
                            r = oy;
                            th = pi / 2 - pi / 4 * (ox / oy);
                        }
                        x = r * std::cos(th);
                        y = r * std::sin(th);
                    }
                    const float wi[3] = {x, y, std::sqrt(std::max(0.f, 1 - x * x - y * y))};
                    const float co = std::fabs(wo[2]), ci = std::fabs(wi[2]);
                    if (co == 0.f || ci == 0.f) continue;
                    float h[3] = {wo[0] + wi[0], wo[1] + wi[1], wo[2] + wi[2]};
                    const float hl = std::sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
                    const float hz = h[2] / hl, inv = 1.f / a, sin2 = std::max(0.f, 1 - hz * hz);
                    const float D = (2 + inv) * std::pow(sin2, 0.5f * inv) / (2 * pi);
                    sum += D / (4 * (ci + co - ci * co)) * pi;
                }
            t[size_t(ia) * nMu + im] = float(sum / (nS * nS));
        }
    }
    return t;
}

namespace {

// Macro cells per axis of a grid's majorant table: one per 8 voxels, at most 32.
static int macro_cells(int n) { return std::max(1, std::min(32, (n + 7) / 8)); }

// Per macro cell, the largest voxel among those the trilinear lookup can touch for a point inside
// the cell (voxel centres within one voxel of it), widened by one more voxel on every side so that
// rounding in the lookup's or the walk's coordinates can never leave a point under its bound.
static std::vector<float> macro_majorants(const float *d, int nx, int ny, int nz, int *mx, int *my, int *mz) {
    const int n[3] = {nx, ny, nz};
    int m[3];
    std::vector<int> lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        m[a] = macro_cells(n[a]);
        for (int c = 0; c < m[a]; ++c) {
            double x0 = double(c) * n[a] / m[a] - 0.5, x1 = double(c + 1) * n[a] / m[a] - 0.5;
            lo[a].push_back(std::max(0, int(std::floor(x0)) - 1));
            hi[a].push_back(std::min(n[a] - 1, int(std::floor(x1)) + 2));
        }
    }
    *mx = m[0], *my = m[1], *mz = m[2];
    // Separable running maxima: along x, then y, then z.
    std::vector<float> ax(size_t(m[0]) * ny * nz), ay(size_t(m[0]) * m[1] * nz), az(size_t(m[0]) * m[1] * m[2]);
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int c = 0; c < m[0]; ++c) {
                float v = 0.f;
                for (int x = lo[0][size_t(c)]; x <= hi[0][size_t(c)]; ++x) v = std::max(v, d[(size_t(z) * ny + y) * nx + x]);
                ax[(size_t(z) * ny + y) * m[0] + c] = v;
            }
    for (int z = 0; z < nz; ++z)
        for (int c = 0; c < m[1]; ++c)
            for (int x = 0; x < m[0]; ++x) {
                float v = 0.f;
                for (int y = lo[1][size_t(c)]; y <= hi[1][size_t(c)]; ++y) v = std::max(v, ax[(size_t(z) * ny + y) * m[0] + x]);
                ay[(size_t(z) * m[1] + c) * m[0] + x] = v;
            }
    for (int c = 0; c < m[2]; ++c)
        for (int y = 0; y < m[1]; ++y)
            for (int x = 0; x < m[0]; ++x) {
                float v = 0.f;
                for (int z = lo[2][size_t(c)]; z <= hi[2][size_t(c)]; ++z) v = std::max(v, ay[(size_t(z) * m[1] + y) * m[0] + x]);
                az[(size_t(c) * m[1] + y) * m[0] + x] = v;
            }
    return az;
}

// Image textures: the descriptors, their texels concatenated, the per-material indices and the
// RGB -> spectrum table.
void upload_textures(const prgpu::SceneExt *ext, SceneCache &cache, DevScene &d, cudaStream_t s) {
    d.textures = nullptr;
    d.matTex = nullptr;
    d.rgbZ = d.rgbCoeffs = nullptr;
    d.texCount = 0;
    d.texNodes = nullptr;
    const int32_t n = ext && ext->textures ? ext->textureCount : 0;
    const int32_t nm = ext && ext->materialTextures ? ext->materialTextureCount : 0;
    const int32_t nn = ext && ext->textureNodes ? ext->textureNodeCount : 0;
    bool used = false;
    for (int32_t i = 0; i < nm; ++i) {
        const prgpu::MaterialTextures &x = ext->materialTextures[i];
        used = used || (n > 0 && (x.reflectance >= 0 || x.normalMap >= 0 || x.bumpMap >= 0)) ||
               (nn > 0 && (x.reflectanceNode >= 0 || x.bumpNode >= 0 || x.roughnessNodeU >= 0 || x.roughnessNodeV >= 0 ||
                           x.coatRoughnessNode >= 0 || x.thicknessNode >= 0 || x.coatAlbedoNode >= 0 ||
                           x.sheenColorNode >= 0 || x.sheenRoughnessNode >= 0 || x.etaNode >= 0));
    }
    if (!used) return;
    size_t total = 0;
    for (int32_t k = 0; k < n; ++k) total += size_t(ext->textures[k].width) * ext->textures[k].height * 3;
    cache.texData.ensure(total * sizeof(float));
    std::vector<DevTex> t(static_cast<size_t>(n));
    size_t off = 0;
    for (int32_t k = 0; k < n; ++k) {
        const prgpu::ImageTextureDesc &x = ext->textures[k];
        const size_t m = size_t(x.width) * x.height * 3;
        PRB_CUDA(cudaMemcpyAsync(cache.texData.as<float>() + off, x.rgb, m * sizeof(float), cudaMemcpyHostToDevice, s));
        DevTex &g = t[size_t(k)];
        g.w = x.width;
        g.h = x.height;
        g.rgb = cache.texData.as<float>() + off;
        g.wrap = int(x.wrap);
        g.flipV = x.flipV ? 1 : 0;
        g.su = x.scaleU, g.sv = x.scaleV, g.ou = x.offsetU, g.ov = x.offsetV;
        g.scale[0] = x.rgbScale[0], g.scale[1] = x.rgbScale[1], g.scale[2] = x.rgbScale[2];
        off += m;
    }
    std::vector<int4> mt(static_cast<size_t>(5 * nm));
    for (int32_t i = 0; i < nm; ++i) {
        const prgpu::MaterialTextures &x = ext->materialTextures[i];
        int sbits, bbits;
        std::memcpy(&sbits, &x.normalStrength, sizeof(sbits));
        std::memcpy(&bbits, &x.bumpScale, sizeof(bbits));
        const bool img = n > 0, trees = nn > 0;
        auto tree = [&](int32_t v) { return trees ? v : -1; };
        mt[size_t(5 * i)] = make_int4(img ? x.reflectance : -1, img ? x.normalMap : -1, sbits, x.normalFlipGreen ? 1 : 0);
        mt[size_t(5 * i + 1)] = make_int4(img ? x.bumpMap : -1, x.bumpChannel, bbits, tree(x.reflectanceNode));
        mt[size_t(5 * i + 2)] = make_int4(tree(x.bumpNode), tree(x.roughnessNodeU), tree(x.roughnessNodeV),
                                          tree(x.sheenRoughnessNode));
        mt[size_t(5 * i + 3)] = make_int4(tree(x.coatRoughnessNode), tree(x.thicknessNode), tree(x.coatAlbedoNode),
                                          tree(x.sheenColorNode));
        mt[size_t(5 * i + 4)] = make_int4(tree(x.etaNode), tree(x.kNode), 0, 0);
    }
    if (n > 0) put(cache.textures, t.data(), t.size(), s);
    put(cache.matTex, mt.data(), mt.size(), s);
    if (nn > 0) put(cache.texNodes, ext->textureNodes, size_t(nn), s);
    if (ext->rgbToSpectrum) {
        const size_t tableFloats = 64 + size_t(3) * 64 * 64 * 64 * 3;
        put(cache.rgbTable, ext->rgbToSpectrum, tableFloats, s);
    }
    PRB_CUDA(cudaStreamSynchronize(s));
    d.textures = n > 0 ? cache.textures.as<DevTex>() : nullptr;
    d.matTex = cache.matTex.as<int4>();
    d.texNodes = nn > 0 ? cache.texNodes.as<prgpu::TextureNode>() : nullptr;
    d.rgbZ = ext->rgbToSpectrum ? cache.rgbTable.as<float>() : nullptr;
    d.rgbCoeffs = d.rgbZ ? d.rgbZ + 64 : nullptr;
    d.texCount = n;
}

// Spot, distant and goniometric lights: the descriptor table and the profiles, concatenated.
void upload_deltas(const prgpu::SceneExt *ext, SceneCache &cache, DevScene &d, cudaStream_t s) {
    d.deltas = nullptr;
    d.deltaCount = 0;
    const int32_t n = ext && ext->deltaLights ? ext->deltaLightCount : 0;
    if (n <= 0) return;
    std::vector<DevDelta> t(static_cast<size_t>(n));
    std::vector<float> prof;
    std::vector<size_t> off(static_cast<size_t>(n), 0);
    for (int32_t k = 0; k < n; ++k) {
        const prgpu::DeltaLightDesc &l = ext->deltaLights[k];
        DevDelta &g = t[size_t(k)];
        g.type = int(l.type);
        g.spectrum = l.spectrum;
        g.scale = l.scale;
        g.pmf = l.pmf;
        g.pos = mk(l.position.x, l.position.y, l.position.z);
        V3 dir = mk(l.direction.x, l.direction.y, l.direction.z);
        float len = std::sqrt(dir.x * dir.x + dir.y * dir.y + dir.z * dir.z);
        g.dir = len > 0.f ? mk(dir.x / len, dir.y / len, dir.z / len) : mk(0.f, 0.f, 1.f);
        g.cosStart = l.cosFalloffStart;
        g.cosEnd = l.cosFalloffEnd;
        g.fx = mk(l.frame[0], l.frame[1], l.frame[2]);
        g.fy = mk(l.frame[3], l.frame[4], l.frame[5]);
        g.fz = mk(l.frame[6], l.frame[7], l.frame[8]);
        g.nV = l.nV;
        g.nH = l.nH;
        g.profile = nullptr;
        if (l.type == prgpu::DeltaGoniometric) {
            off[size_t(k)] = prof.size();
            const size_t m = size_t(l.nV) + size_t(l.nH) + size_t(l.nV) * size_t(l.nH);
            prof.insert(prof.end(), l.profile, l.profile + m);
        }
    }
    if (!prof.empty()) {
        put(cache.deltaProfiles, prof.data(), prof.size(), s);
        for (int32_t k = 0; k < n; ++k)
            if (t[size_t(k)].type == prgpu::DeltaGoniometric) t[size_t(k)].profile = cache.deltaProfiles.as<float>() + off[size_t(k)];
    }
    put(cache.deltas, t.data(), t.size(), s);
    PRB_CUDA(cudaStreamSynchronize(s));
    d.deltas = cache.deltas.as<DevDelta>();
    d.deltaCount = n;
}

// The image environment's texels and its sampling distribution (EnvironmentLight's constructor,
// light.cpp:217-236, with a spectral luminance in place of the RGB one; Distribution2D,
// sampling.cpp:44-67). Rows are Distribution1D CDFs normalised to 1 (unless all zero).
void upload_env(const prgpu::SceneExt *ext, const prgpu::SceneDesc *sd, SceneCache &cache, DevScene &d,
                cudaStream_t s) {
    d.envMap = DevEnvMap{};
    d.sun = DevSun{};
    d.sun.spectrum = -1;
    if (ext && ext->sun) {
        const prgpu::SunDesc &u = *ext->sun;
        float l = std::sqrt(u.direction.x * u.direction.x + u.direction.y * u.direction.y + u.direction.z * u.direction.z);
        V3 z = mk(u.direction.x / l, u.direction.y / l, u.direction.z / l);
        // Orthonormal frame around z (Duff et al. 2017).
        float sg = std::copysign(1.f, z.z), a = -1.f / (sg + z.z), b = z.x * z.y * a;
        d.sun.x = mk(1.f + sg * z.x * z.x * a, sg * b, -sg * z.x);
        d.sun.y = mk(b, sg + z.y * z.y * a, -z.y);
        d.sun.z = z;
        d.sun.cosMax = u.cosThetaMax;
        d.sun.spectrum = u.spectrum;
        d.sun.scale = u.scale;
        d.sun.pmf = u.pmf;
    }
    upload_deltas(ext, cache, d, s);
    upload_textures(ext, cache, d, s);
    if (!(ext && ext->envMap)) return;
    const prgpu::EnvMapDesc &e = *ext->envMap;
    const int w = e.width, h = e.height;
    const size_t n = size_t(w) * h;
    put(cache.envTexels, reinterpret_cast<const float4 *>(e.texels), n, s);
    // Luminance of each texel: its spectrum times the illuminant against CIE y over the table.
    std::vector<float> func(n), rowCdf(static_cast<size_t>(h) * (w + 1)), rowInt(static_cast<size_t>(h)),
        marg(static_cast<size_t>(h) + 1);
    const float *ybar = sd->cie ? sd->cie + prgpu::kSpectrumSamples : nullptr;
    for (int v = 0; v < h; ++v) {
        const float sinTheta = std::sin(3.14159265358979f * (float(v) + 0.5f) / float(h));
        for (int u = 0; u < w; ++u) {
            const float *t = e.texels + 4 * (size_t(v) * w + u);
            double y = 0.0;
            for (int i = 0; i < prgpu::kSpectrumSamples; ++i) {
                float l = prgpu::kSpectrumMin + prgpu::kSpectrumStep * float(i);
                float il = e.illuminant >= 0 ? sd->spectra[e.illuminant].v[i] : 1.f;
                y += double(texel_value(t, l)) * il * (ybar ? ybar[i] : 1.f);
            }
            func[size_t(v) * w + u] = float(std::max(0.0, y)) * sinTheta + 1e-6f;
        }
        float *cdf = rowCdf.data() + size_t(v) * (w + 1);
        cdf[0] = 0.f;
        for (int u = 0; u < w; ++u) cdf[u + 1] = cdf[u] + func[size_t(v) * w + u] / float(w);
        rowInt[size_t(v)] = cdf[w];
        for (int u = 1; u <= w; ++u) cdf[u] = cdf[w] > 0.f ? cdf[u] / cdf[w] : float(u) / float(w);
    }
    marg[0] = 0.f;
    for (int v = 0; v < h; ++v) marg[size_t(v) + 1] = marg[size_t(v)] + rowInt[size_t(v)] / float(h);
    const float margInt = marg[size_t(h)];
    for (int v = 1; v <= h; ++v) marg[size_t(v)] = margInt > 0.f ? marg[size_t(v)] / margInt : float(v) / float(h);
    std::vector<float> dist;
    dist.reserve(func.size() + rowCdf.size() + rowInt.size() + marg.size());
    dist.insert(dist.end(), func.begin(), func.end());
    dist.insert(dist.end(), rowCdf.begin(), rowCdf.end());
    dist.insert(dist.end(), rowInt.begin(), rowInt.end());
    dist.insert(dist.end(), marg.begin(), marg.end());
    put(cache.envDist, dist.data(), dist.size(), s);
    PRB_CUDA(cudaStreamSynchronize(s));
    const float *base = cache.envDist.as<float>();
    DevEnvMap &m = d.envMap;
    m.w = w;
    m.h = h;
    m.texels = cache.envTexels.as<float4>();
    m.func = base;
    m.rowCdf = base + func.size();
    m.rowInt = m.rowCdf + rowCdf.size();
    m.margCdf = m.rowInt + rowInt.size();
    m.margInt = margInt;
    m.illuminant = e.illuminant;
    m.scale = e.scale;
    m.pmf = e.pmf;
    const float rad = e.rotationDeg * 3.14159265358979f / 180.f;
    m.rc = std::cos(rad);
    m.rs = std::sin(rad);
}

} // namespace

bool upload_scene(DeviceState &ds, const prgpu::SceneDesc *sd, const prgpu::SceneExt *ext, SceneCache &cache,
                  std::string *err) {
    if (!validate(sd, ext, err)) return false;
    uint64_t key = scene_key(sd, ext);
    DevScene &d = cache.ds;
    if (!cache.valid || cache.key != key) {
        HostAccel h;
        if (!convert_bvh(sd->nodes, sd->nodeCount, sd->primOrder, sd->primCount, PrimitiveSource{sd->prims}, &h, err))
            return false;
        cudaStream_t s = ds.stream;
        cache.accel.upload(h, s);
        put(cache.prims, sd->prims, size_t(sd->primCount), s);
        std::vector<uint8_t> cls(size_t(std::max(1, sd->primCount)), uint8_t(kClassOther));
        for (int32_t i = 0; i < sd->primCount; ++i) {
            uint32_t t = sd->materials[sd->prims[i].material].type;
            cls[size_t(i)] = uint8_t(t == prgpu::MatDiffuse      ? kClassDiffuse
                                     : t == prgpu::MatConductor  ? kClassConductor
                                     : t == prgpu::MatDielectric ? kClassDielectric
                                                                 : kClassOther);
            const prgpu::Material &mi = sd->materials[sd->prims[i].material];
            if (mi.sheenWeight > 0 && mi.sheenColor >= 0) cls[size_t(i)] = uint8_t(kClassOther);
            if (t == prgpu::MatInterface) cls[size_t(i)] |= kTransparentBit;
        }
        put(cache.primClass, cls.data(), cls.size(), s);
        std::vector<LeafPrim> walls;
        for (const LeafPrim &lp : h.prims) {
            int32_t id;
            std::memcpy(&id, &lp.v0.w, sizeof(id));
            if (id >= 0 && id < sd->primCount && (cls[size_t(id)] & kTransparentBit)) walls.push_back(lp);
        }
        cache.wallCount = walls.size() <= size_t(kMaxWallList) ? int(walls.size()) : -1;
        if (cache.wallCount > 0) put(cache.walls, walls.data(), walls.size(), s);
        cache.hasSheen = false;
        for (int32_t i = 0; i < sd->materialCount; ++i)
            if (sd->materials[i].sheenWeight > 0 && sd->materials[i].sheenColor >= 0) cache.hasSheen = true;
        if (cache.hasSheen) {
            std::vector<float> table = sd->sheenAlbedo
                                           ? std::vector<float>(sd->sheenAlbedo, sd->sheenAlbedo + prgpu::kSheenAlpha * prgpu::kSheenMu)
                                           : sheen_albedo_table();
            put(cache.sheen, table.data(), table.size(), s);
        }
        put(cache.mats, sd->materials, size_t(sd->materialCount), s);
        put(cache.lights, sd->lights, size_t(sd->lightCount), s);
        put(cache.spectra, sd->spectra, size_t(sd->spectrumCount), s);
        put(cache.media, sd->media, size_t(sd->mediumCount), s);
        put(cache.filterCdf, sd->filter.cdf, size_t(prgpu::kFilterBins + 1), s);
        int32_t nb = (ext && ext->lightBVHNodeCount > 0) ? ext->lightBVHNodeCount : 0;
        std::vector<int> leafOf(size_t(std::max(1, sd->lightCount)), -1);
        for (int32_t i = 0; i < nb; ++i)
            if (ext->lightBVH[i].light >= 0) leafOf[size_t(ext->lightBVH[i].light)] = i;
        if (nb) put(cache.lbvh, ext->lightBVH, size_t(nb), s);
        // Grid media: the density grids concatenated in one buffer, plus the descriptor table.
        int32_t ng = (ext && ext->gridMediumCount > 0) ? ext->gridMediumCount : 0;
        std::vector<DevGrid> grids(size_t(std::max(1, ng)));
        size_t total = 0;
        for (int32_t k = 0; k < ng; ++k) {
            const prgpu::GridMediumDesc &g = ext->gridMedia[k];
            if (g.field == prgpu::GridNoise) total += 1;
            else if (g.field == prgpu::GridIndexed) total += size_t(g.nx) * g.ny * g.nz + 1;
            else total += size_t(g.nx) * g.ny * g.nz + size_t(macro_cells(g.nx)) * macro_cells(g.ny) * macro_cells(g.nz);
        }
        cache.gridData.ensure(std::max<size_t>(1, total) * sizeof(float));
        size_t off = 0;
        for (int32_t k = 0; k < ng; ++k) {
            const prgpu::GridMediumDesc &g = ext->gridMedia[k];
            DevGrid &dg = grids[size_t(k)];
            std::memcpy(dg.w2m, g.worldToMedium, sizeof(dg.w2m));
            dg.bmin[0] = g.boundsMin.x, dg.bmin[1] = g.boundsMin.y, dg.bmin[2] = g.boundsMin.z;
            dg.bmax[0] = g.boundsMax.x, dg.bmax[1] = g.boundsMax.y, dg.bmax[2] = g.boundsMax.z;
            dg.scale = g.scale;
            dg.g = std::min(0.99f, std::max(-0.99f, g.g));
            dg.sigmaA = g.sigmaA;
            dg.sigmaS = g.sigmaS;
            dg.noise = g.field == prgpu::GridNoise ? 1 : 0;
            dg.boundless = 0;
            if (dg.noise) {
                // One macro cell over the bounds with the field's maximum density (1). Empty bounds
                // (Bounds3f::IsEmpty, math.h:212: min > max on an axis): no bounds at all, and no
                // falloff (NoiseField::Density, medium.cpp:168-177); the zeroed box makes the
                // macro-cell walk one cell over the whole segment.
                if (g.boundsMin.x > g.boundsMax.x || g.boundsMin.y > g.boundsMax.y || g.boundsMin.z > g.boundsMax.z) {
                    dg.boundless = 1;
                    for (int a = 0; a < 3; ++a) dg.bmin[a] = dg.bmax[a] = 0.f;
                }
                dg.nx = dg.ny = dg.nz = 0;
                dg.density = nullptr;
                dg.maxDensity = std::max(1.f, std::isfinite(g.maxDensity) ? g.maxDensity : 1.f);
                dg.mx = dg.my = dg.mz = 1;
                dg.noiseOctaves = g.noiseOctaves;
                dg.noiseFalloff = g.noiseFalloff && !dg.boundless ? 1 : 0;
                dg.noiseFrequency = g.noiseFrequency;
                dg.noiseThreshold = g.noiseThreshold;
                dg.noiseSharpness = g.noiseSharpness;
                std::memcpy(dg.noiseOffset, g.noiseOffset, sizeof(dg.noiseOffset));
                dg.majorant = cache.gridData.as<float>() + off;
                PRB_CUDA(cudaMemcpyAsync(const_cast<float *>(dg.majorant), &dg.maxDensity, sizeof(float),
                                         cudaMemcpyHostToDevice, s));
                PRB_CUDA(cudaStreamSynchronize(s));
                off += 1;
                continue;
            }
            size_t n = size_t(g.nx) * g.ny * g.nz;
            dg.nx = g.nx, dg.ny = g.ny, dg.nz = g.nz;
            if (g.field == prgpu::GridIndexed) {
                // Raw voxels (non-finite ones read as 0; the trilinear result is clamped at 0) and
                // one macro cell with the largest voxel.
                dg.indexed = 1;
                std::memcpy(dg.org, g.indexOrigin, sizeof(dg.org));
                std::vector<float> raw(g.density, g.density + n);
                float mx = 0.f;
                for (float &v : raw) {
                    if (!std::isfinite(v)) v = 0.f;
                    mx = std::max(mx, v);
                }
                dg.maxDensity = std::max(mx, std::isfinite(g.maxDensity) ? g.maxDensity : 0.f);
                dg.mx = dg.my = dg.mz = 1;
                dg.density = cache.gridData.as<float>() + off;
                dg.majorant = dg.density + n;
                PRB_CUDA(cudaMemcpyAsync(const_cast<float *>(dg.density), raw.data(), n * sizeof(float),
                                         cudaMemcpyHostToDevice, s));
                PRB_CUDA(cudaMemcpyAsync(const_cast<float *>(dg.majorant), &dg.maxDensity, sizeof(float),
                                         cudaMemcpyHostToDevice, s));
                PRB_CUDA(cudaStreamSynchronize(s));
                off += n + 1;
                continue;
            }
            // Negative or non-finite voxels read as 0, as pr::VoxelGridField does (medium.cpp:108-115).
            float mx = 0.f;
            for (size_t i = 0; i < n; ++i)
                if (std::isfinite(g.density[i]) && g.density[i] > mx) mx = g.density[i];
            dg.maxDensity = g.maxDensity > mx ? g.maxDensity : mx;
            dg.scale = g.scale;
            dg.g = std::min(0.99f, std::max(-0.99f, g.g));
            dg.sigmaA = g.sigmaA;
            dg.sigmaS = g.sigmaS;
            dg.density = cache.gridData.as<float>() + off;
            std::vector<float> clean(g.density, g.density + n);
            for (float &v : clean)
                if (!std::isfinite(v) || v < 0.f) v = 0.f;
            std::vector<float> maj = macro_majorants(clean.data(), g.nx, g.ny, g.nz, &dg.mx, &dg.my, &dg.mz);
            dg.majorant = dg.density + n;
            PRB_CUDA(cudaMemcpyAsync(const_cast<float *>(dg.density), clean.data(), n * sizeof(float),
                                     cudaMemcpyHostToDevice, s));
            PRB_CUDA(cudaMemcpyAsync(const_cast<float *>(dg.majorant), maj.data(), maj.size() * sizeof(float),
                                     cudaMemcpyHostToDevice, s));
            PRB_CUDA(cudaStreamSynchronize(s));
            off += n + maj.size();
        }
        put(cache.grids, grids.data(), grids.size(), s);
        d.grids = cache.grids.as<DevGrid>();
        d.gridCount = ng;
        upload_env(ext, sd, cache, d, s);
        put(cache.lightLeaf, leafOf.data(), leafOf.size(), s);
        PRB_CUDA(cudaStreamSynchronize(s));
        cache.hasSpheres = false;
        for (int32_t i = 0; i < sd->primCount; ++i)
            if (sd->prims[i].type == prgpu::PrimSphere) cache.hasSpheres = true;
        cache.key = key;
        cache.valid = true;
        cache.deviceBytes = cache.accel.bytes + int64_t(sd->primCount) * int64_t(sizeof(prgpu::Primitive));
        d.nodes = cache.accel.nodes.as<WNode>();
        d.qnodes = cache.accel.qnodes.as<QNode>();
        d.leaves = cache.accel.prims.as<LeafPrim>();
        d.root = cache.accel.root;
        d.prims = cache.prims.as<prgpu::Primitive>();
        d.primClass = cache.primClass.as<uint8_t>();
        d.sheenTable = cache.hasSheen ? cache.sheen.as<float>() : nullptr;
        d.walls = cache.wallCount > 0 ? cache.walls.as<LeafPrim>() : nullptr;
        d.wallCount = cache.wallCount;
        d.mats = cache.mats.as<prgpu::Material>();
        d.lights = cache.lights.as<prgpu::Light>();
        d.spectra = cache.spectra.as<float>();
        d.media = cache.media.as<prgpu::Medium>();
        d.filterCdf = cache.filterCdf.as<float>();
        d.lbvh = nb ? cache.lbvh.as<prgpu::LightBVHNode>() : nullptr;
        d.lightLeaf = cache.lightLeaf.as<int>();
        d.lbvhCount = nb;
    }
    // Per-call scalars (cheap; not part of the device copy).
    d.mediumCount = sd->mediumCount;
    d.lightCount = sd->lightCount;
    d.cameraMedium = sd->cameraMedium;
    d.envSpectrum = sd->envSpectrum;
    d.envScale = sd->envScale;
    d.worldRadius = sd->worldRadius;
    d.cam = sd->camera;
    d.norm = sd->cieYIntegral > 0 ? 1.f / (4.f * sd->cieYIntegral) : 0.f;
    d.hasInterfaces = 0;
    d.hasFull = 0;
    for (int32_t i = 0; i < sd->materialCount; ++i) {
        const prgpu::Material &m = sd->materials[i];
        if (m.type == prgpu::MatInterface) d.hasInterfaces = 1;
        if (m.type == prgpu::MatCoatedDiffuse || m.type == prgpu::MatCoatedConductor ||
            (m.sheenWeight > 0 && m.sheenColor >= 0))
            d.hasFull = 1;
    }
    d.filterType = sd->filter.type;
    d.filterRadius = sd->filter.radius;
    d.filterSigma = sd->filter.sigma;
    d.filterNorm = sd->filter.norm;
    if (d.lbvhCount > 0) {
        d.lbvhProb = ext->lightBVHProb > 0 && ext->lightBVHProb <= 1 ? ext->lightBVHProb : 1.f;
        d.envPmf = sd->envSpectrum >= 0 ? 1.f - d.lbvhProb : 0.f;
    } else {
        d.lbvhProb = 0.f;
        d.envPmf = sd->envPmf;
    }
    return true;
}

} // namespace prb
