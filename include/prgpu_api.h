// prgpu_api.h -- the C ABI of libprender_gpu.so, the B200 (sm_100a) path-tracing module.
//
// The first part restates, layout for layout, the plain-data interface that PRender's host
// (src/integrators/gpu_path.cpp) hands its GPU module, so that this library is a drop-in for
// prender_gpu: the reference declares it in src/gpu/gpu_api.h:15-173 and checks
// prgpu_api_version() == 4 before use (src/integrators/gpu_path.cpp:59-65). Every struct below
// must stay byte-identical to those layouts; static_asserts in the implementation pin sizes and
// offsets.
//
// The second part (PRGPU extension, version 5) adds entry points the v4 interface cannot
// express: a ray-query service over a caller BVH, an FP64 film with fixed-order accumulation,
// light-BVH next-event estimation, device-resident handles for benchmarking, and run
// statistics. A v4 caller never sees them.
//
// All pointers are caller-owned host memory unless the name says "device"; they need only be
// valid for the duration of the call. Entry points never throw; they return 0 on success and
// otherwise write a NUL-terminated message into err (when err != nullptr and errLen > 0).
#pragma once

#include <cstdint>

#if defined(_WIN32)
#define PRGPU_API extern "C" __declspec(dllexport)
#else
#define PRGPU_API extern "C" __attribute__((visibility("default")))
#endif

namespace prgpu {

// --------------------------------------------------------------------------------------------
// v4 plain-data layouts (src/gpu/gpu_api.h:17-162)

constexpr int kApiVersion = 4;          // gpu_api.h:17
constexpr int kExtVersion = 5;          // this library's extension level
constexpr int kGuideParams = 23552;     // weights of the path-guiding network
constexpr int kSpectrumSamples = 95;    // 360..830 nm every 5 nm, linear interpolation (gpu_api.h:19-21)
constexpr float kSpectrumMin = 360.f, kSpectrumStep = 5.f;
constexpr int kFilterBins = 64;         // pixel-filter CDF bins (gpu_api.h:22-23)
constexpr int kSheenMu = 32, kSheenAlpha = 16;  // sheen albedo table (gpu_api.h:24-25)

struct Float3 {
    float x, y, z;
};

struct Spectrum {
    float v[kSpectrumSamples];
};

// Flattened binary BVH node, depth-first: an interior node's first child follows it, `offset`
// names the second child; a leaf covers primOrder[offset .. offset+nPrims). (gpu_api.h:35-40)
struct BVHNode {
    Float3 bmin, bmax;
    int32_t offset;
    uint16_t nPrims;  // 0 = interior
    uint8_t axis, pad;
};

enum PrimType : uint32_t { PrimTriangle = 0, PrimSphere = 1 };

// One primitive: a triangle (p0..p2, optional vertex normals n0..n2 -- n0 == 0 means flat -- and
// uvs) or a sphere (centre p0, radius r, flip = inward normals). (gpu_api.h:44-56)
struct Primitive {
    uint32_t type;
    int32_t material;
    int32_t light;                        // area light index or -1
    int32_t mediumInside, mediumOutside;  // medium on each side, -1 = vacuum
    uint32_t pad;
    Float3 p0, p1, p2;
    Float3 n0, n1, n2;
    float u0, v0, u1, v1, u2, v2;
    float r;
    uint32_t flip;
};

enum MaterialType : uint32_t {
    MatDiffuse = 0, MatConductor = 1, MatDielectric = 2, MatBlack = 3, MatInterface = 4,
    MatCoatedDiffuse = 5, MatCoatedConductor = 6
};

// Material parameters; spectra are indices into SceneDesc::spectra, -1 = none. (gpu_api.h:61-81)
struct Material {
    uint32_t type;
    int32_t albedo, albedoB;  // reflectance (diffuse / artist conductor); checker second colour
    float checkerScale;       // checker frequency in uv, 0 = plain
    int32_t eta, k;           // conductor n, k; dielectric IOR
    float alphaX, alphaY;     // GGX alpha (roughness^2); max < 1e-3 = smooth
    uint32_t dispersive;      // IOR varies with wavelength -> secondary wavelengths terminate
    uint32_t thin;
    int32_t coatEta;
    float coatAlpha, thickness, coatG;
    int32_t coatAlbedo;
    uint32_t coatDispersive;
    int32_t coatMaxDepth, coatSamples;
    int32_t sheenColor;
    float sheenRoughness, sheenWeight;
    uint32_t pad;
};

// Homogeneous medium: sigma = spectrum * scale, Henyey-Greenstein g. (gpu_api.h:84-87)
struct Medium {
    int32_t sigmaA, sigmaS;
    float scale, g;
};

enum FilterType : uint32_t { FilterBox = 0, FilterGaussian = 1, FilterBlackmanHarris = 2 };

struct Filter {  // gpu_api.h:91-95
    uint32_t type;
    float radius, sigma, norm;
    float cdf[kFilterBins + 1];
};

enum LightType : uint32_t { LightArea = 0, LightPoint = 1 };

struct Light {  // gpu_api.h:99-110
    uint32_t type;
    int32_t primitive;  // area: emitting primitive
    int32_t spectrum;   // radiance (area) or intensity (point)
    float scale;
    Float3 position;    // point light
    uint32_t twoSided;
    float cosPower;
    float area;
    float pmf;          // power-based selection probability
    uint32_t pad;
};

struct Camera {  // gpu_api.h:112-118
    float cameraToWorld[12];  // row-major 3x4
    float tanHalfFov, aspect;
    float lensRadius, focalDistance;
    int32_t width, height, margin;
    uint32_t pad;
};

struct SceneDesc {  // gpu_api.h:120-146
    int32_t apiVersion;
    const BVHNode *nodes;
    int32_t nodeCount;
    const int32_t *primOrder;
    const Primitive *prims;
    int32_t primCount;
    const Material *materials;
    int32_t materialCount;
    const Light *lights;
    int32_t lightCount;
    const Spectrum *spectra;
    int32_t spectrumCount;
    const Medium *media;
    int32_t mediumCount;
    int32_t cameraMedium;
    int32_t envSpectrum;
    float envScale;
    float envPmf;
    Float3 worldCenter;
    float worldRadius;
    Camera camera;
    Filter filter;
    const float *sheenAlbedo;  // kSheenAlpha * kSheenMu
    const float *cie;          // 3 x kSpectrumSamples
    float cieYIntegral;
};

struct RenderParams {  // gpu_api.h:148-154
    int32_t spp;
    int32_t firstSample;
    uint64_t seed;
    int32_t maxDepth;       // <= 0: unlimited (Russian roulette)
    float clampLuminance;   // 0 = off
};

struct DeviceInfo {  // gpu_api.h:156-162
    char name[256];
    uint64_t globalMemory;
    int32_t computeUnits;
    int32_t isGpu;
    char backend[32];
};

// --------------------------------------------------------------------------------------------
// Extension (v5) plain-data layouts. No counterpart in src/gpu/gpu_api.h.

// A ray for the ray-query service: origin, tMax, direction (32 bytes; 16-byte aligned pairs).
struct Ray {
    Float3 o;
    float tMax;
    Float3 d;
    float pad;
};

// Light-BVH node for importance-based next-event estimation, the flattened form of
// pr::BVHLightSampler's tree (src/lights/light_bvh.h:23-35, built as in light_bvh.cpp:117-177).
// Interior nodes: first child follows, child1 names the second; leaves: light >= 0 (index into
// SceneDesc::lights). parent = -1 at the root.
struct LightBVHNode {
    Float3 bmin, bmax;
    Float3 w;             // emission cone axis
    float phi;            // power bound
    float cosThetaO, cosThetaE;
    int32_t twoSided;
    int32_t child1, light, parent;
    int32_t pad[2];
};

// Heterogeneous medium: sigma(p, lambda) = density(p) * spectrum(lambda) * scale, Henyey-Greenstein
// g, with a voxel density grid sampled trilinearly at cell centres over `bounds` in medium space
// (pr::GridMedium over a pr::VoxelGridField, src/media/medium.h:93-167, medium.cpp:117-128).
// Distances are sampled by spectral tracking and shadow transmittance by ratio tracking against a
// global majorant maxDensity * max(sigma_t) (medium.cpp:205-285). Media are referenced from
// Primitive::mediumInside/Outside and SceneDesc::cameraMedium with indices mediumCount + k.
// field = GridNoise replaces the voxels by pr::NoiseField (medium.h:119-133, medium.cpp:168-177):
// density = clamp((n - threshold) * sharpness, 0, 1) with n = 0.5 + 0.7 fBm((p + offset) *
// frequency) of improved Perlin noise, faded by 1 - |2 (p - min) / (max - min) - 1|^2 when falloff
// is set; 0 outside the bounds; the majorant is 1 unless maxDensity says more. Empty bounds
// (boundsMin > boundsMax on an axis, as an unset pr::Bounds3f) mean no bounds: the field fills
// every finite segment and has no falloff (GridMedium::Clip, medium.cpp:182-188).
// field = GridIndexed takes the voxels of an index-space grid: a NanoVDB float grid densified by
// the caller (pr::NanoVDBField, media/nanovdb_field.cpp:17-46). Medium space is then the grid's
// index space (worldToMedium = the grid's world-to-index map after the medium's own transform);
// voxel (x, y, z) of `density` sits at the integer index coordinate indexOrigin + (x, y, z), the
// density is trilinear between voxel centres, 0 beyond the array (the grid's background) and
// clamped at 0; bounds (the grid's world box in index space) clip the segments; the majorant is
// the largest voxel.
enum GridField : uint32_t { GridVoxels = 0, GridNoise = 1, GridIndexed = 2 };
struct GridMediumDesc {
    int32_t sigmaA, sigmaS;     // spectrum indices
    float scale, g;
    float worldToMedium[12];    // affine, row-major 3x4
    Float3 boundsMin, boundsMax;
    int32_t nx, ny, nz;
    float maxDensity;           // >= every voxel; 0 = computed from the data
    const float *density;       // nx * ny * nz floats, x fastest: index (z * ny + y) * nx + x
    uint32_t field;             // GridField
    int32_t noiseOctaves;       // [1, 32]
    float noiseFrequency, noiseThreshold, noiseSharpness;
    uint32_t noiseFalloff;
    float noiseOffset[3];
    int32_t indexOrigin[3];     // GridIndexed
};

// Image environment light (pr::EnvironmentLight with a map, src/lights/light.cpp:217-297), as a
// latitude-longitude map with +y up (uv of a direction by DirToEquirect, light.h:292-297).
// Texels hold the sigmoid-polynomial spectra the reference's RGB uplift produces
// (RGBUnboundedSample, src/core/rgb2spec.cpp:328-336): radiance(lambda) = scale *
// S(c0 lambda^2 + c1 lambda + c2) with S(x) = 1/2 + x / (2 sqrt(1 + x^2)) and lambda in nm,
// times the illuminant spectrum (D65 for RGB illuminants, rgb2spec.cpp:338-343). Lookups are
// bilinear with horizontal wrap; sampling follows a 2D distribution of luminance x sin(theta).
struct EnvMapDesc {
    int32_t width, height;
    const float *texels;      // width * height * 4 floats: c0, c1, c2, scale (row 0 = theta 0)
    int32_t illuminant;       // spectrum index multiplied into every texel, -1 = none
    float scale;
    float rotationDeg;        // rotation of the map about +y (Transform::Rotate, light.cpp:219-220)
    float pmf;                // selection probability of this light in next-event estimation
};

// Sun disk (pr::SunLight, src/lights/sky.cpp:84-109): uniform radiance inside a cone.
struct SunDesc {
    Float3 direction;         // towards the sun (normalised on upload)
    float cosThetaMax;        // cosine of the angular radius
    int32_t spectrum;         // radiance spectrum index
    float scale;
    float pmf;                // selection probability of this light in next-event estimation
};

// Optional extras for prgpu_render_ex (zero-initialise, then set structSize = sizeof(SceneExt)).
// A delta light the v4 light table cannot describe (src/lights/light.h:143-240): a spot light
// (SpotLight, light.cpp:161-192), a distant light (DistantLight, sky.cpp:52-63) or a goniometric
// point light with a type C IES profile (GoniometricLight / IESProfile, sky.cpp:12-26,
// ies.cpp:79-109). Selected with probability pmf alongside the SceneDesc lights and the infinite
// lights (all pmfs together sum to 1).
enum DeltaLightType : uint32_t { DeltaSpot = 0, DeltaDistant = 1, DeltaGoniometric = 2 };
struct DeltaLightDesc {
    uint32_t type;
    int32_t spectrum;        // intensity (spot, goniometric) or irradiance (distant) spectrum index
    float scale;
    float pmf;
    Float3 position;         // spot, goniometric
    Float3 direction;        // spot: cone axis (where it shines); distant: towards the light
    float cosFalloffStart;   // spot: cos of the falloff start and of the cone's half width
    float cosFalloffEnd;
    float frame[9];          // goniometric: profile frame rows x, y, z (z = the profile's nadir)
    int32_t nV, nH;          // goniometric: vertical and horizontal angle counts
    int32_t pad;
    const float *profile;    // goniometric: vAngles[nV], hAngles[nH] (degrees), candela[nH][nV] / peak
};

// An RGB image texture (pr::ImageData + pr::ImageSpectrumTexture, src/materials/texture.h:60-105,
// texture.cpp:8-53): bilinear lookup with a wrap mode, the UV mapping, an RGB scale, and the
// albedo uplift of the looked-up colour through the RGB -> spectrum table.
enum TextureWrap : uint32_t { WrapRepeat = 0, WrapClamp = 1, WrapMirror = 2 };
struct ImageTextureDesc {
    int32_t width, height;
    const float *rgb;        // width * height * 3 linear RGB, row 0 first (pr::Image)
    uint32_t wrap;           // TextureWrap
    uint32_t flipV;          // look up at v' = 1 - v
    float scaleU, scaleV, offsetU, offsetV;  // pr::UVMapping
    float rgbScale[3];
    uint32_t pad;
};

// A node of a procedural texture tree (pr::CheckerSpectrumTexture / CheckerFloatTexture,
// NoiseFloatTexture, MixSpectrumTexture / MixFloatTexture and their constant and image leaves:
// texture.h:35-205). A tree is used either as a spectrum texture (reflectance) or as a float
// texture (bump height, roughness); its root is named by MaterialTextures.
//   TexConstant  spectrum use: a = SceneDesc::spectra index; float use: value
//   TexImage     a = SceneExt::textures index; spectrum use: the looked-up colour times rgbScale,
//                uplifted as an albedo; float use: `channel` (-1 the mean of r, g, b) times
//                rgbScale (the float texture's multiplier in all three components)
//   TexChecker   a where floor(s) + floor(t) is even, else b; (s, t) = uv * scale + offset
//   TexNoise     float use only: fBm of improved Perlin noise at (p + offset) * frequency, p the
//                hit point (flags & TexNoiseWorldSpace) or (u, v, 0); octaves in [1, 32]
//   TexMix       a (1 - t) + b t, t = node `t` (a TexNoise node) clamped to [0, 1]
// Trees are at most 8 nodes deep.
enum TextureNodeType : uint32_t { TexConstant = 0, TexImage = 1, TexChecker = 2, TexNoise = 3, TexMix = 4 };
enum TextureNoiseFlags : uint32_t { TexNoiseTurbulence = 1, TexNoiseWorldSpace = 2 };
struct TextureNode {
    uint32_t type;
    int32_t a, b, t;
    int32_t channel;
    float value;
    float frequency;
    int32_t octaves;
    uint32_t flags;
    float offset[3];
    float scaleU, scaleV, offsetU, offsetV;
};

// Per SceneDesc material: the image texture of its reflectance (diffuse and coated diffuse
// materials, and the artist reflectance of conductors and coated conductors given by reflectance
// rather than n and k: ConductorMaterial::MakeBxDF, material.cpp:90-96), of its tangent-space
// normal map and of its bump (height) map (any material;
// pr::NormalMapParams / BumpMapParams, material.h:30-41, applied as Material::PerturbShading,
// material.cpp:16-60), -1 for none. A height map's texture carries the float texture's
// multiplier in all three rgbScale components. The *Node fields name TextureNode trees instead
// (-1 none); a reflectance or bump tree takes precedence over the image of the same slot, and the
// roughness trees replace the GGX roughness (alpha = clamp(r, 0, 1)^2) of conductor, rough
// dielectric and coated-conductor base lobes, each direction separately. The coat trees replace
// the coat's roughness, thickness and medium albedo (coated materials, MakeCoatTop,
// material.cpp:119-130) and the sheen trees its colour and roughness (Material::GetBSDF,
// material.cpp:5-14).
struct MaterialTextures {
    int32_t reflectance;
    int32_t normalMap;
    float normalStrength;      // scales the map's tangent-plane components
    uint32_t normalFlipGreen;  // the map's green channel points along -v
    int32_t bumpMap;
    int32_t bumpChannel;       // -1 the mean of r, g, b; 0, 1, 2 one channel
    float bumpScale;
    int32_t reflectanceNode;
    int32_t bumpNode;
    int32_t roughnessNodeU;
    int32_t roughnessNodeV;
    int32_t coatRoughnessNode;
    int32_t thicknessNode;
    int32_t coatAlbedoNode;     // spectrum tree
    int32_t sheenColorNode;     // spectrum tree
    int32_t sheenRoughnessNode;
    // Conductor n and k (conductor and coated-conductor base; ConductorMaterial::MakeBxDF,
    // material.cpp:80-92) as spectrum trees of unbounded spectra: their image leaves are uplifted
    // as RGBUnboundedSpectrum (2 max(r, g, b) times the sigmoid of the colour over that scale).
    int32_t etaNode;
    int32_t kNode;
};

struct SceneExt {
    uint32_t structSize;
    int32_t lightBVHNodeCount;      // 0 = power-based light selection (the v4 behaviour)
    const LightBVHNode *lightBVH;
    float lightBVHProb;             // probability of the BVH branch when envSpectrum >= 0 (1 - pInfinite)
    int32_t wavefrontPaths;         // paths in flight per wavefront (0 = library default)
    int32_t blockSize;              // threads per block for the wavefront kernels (0 = default)
    int32_t flags;                  // path guiding: bit 0 sample diffuse vertices with the guide
                                    // network (one-sample MIS with the BSDF), bit 1 train it online
                                    // (one Adam step per wavefront chunk), bit 2 fresh weights first
    int32_t gridMediumCount;
    const GridMediumDesc *gridMedia;
    const EnvMapDesc *envMap;       // null = none
    const SunDesc *sun;             // null = none
    int32_t deltaLightCount;
    int32_t pad;
    const DeltaLightDesc *deltaLights;
    int32_t textureCount;
    int32_t materialTextureCount;   // 0, or SceneDesc::materialCount
    const ImageTextureDesc *textures;
    const MaterialTextures *materialTextures;
    // RGB -> sigmoid-polynomial table (pr::RGBToSpectrumTable, rgb2spec.h:28-46): zNodes[64] then
    // coefficients[3][64][64][64][3]; required when a material has a texture.
    const float *rgbToSpectrum;
    const TextureNode *textureNodes;
    int32_t textureNodeCount;
    int32_t pad2;
    // Measurement tap (null = off): the rays traced for the paths in wavefront slots
    // [0, rayTapPaths) of the call's first chunk (slot = pixel + pixels-per-chunk * sample), for
    // their first rayTapBounces bounces, copied to HOST memory at rayTap as 2 x rayTapBounces x
    // rayTapPaths records of 8 floats (origin, tMax, direction, 1): the closest-hit rays, then the
    // shadow rays (tMax in units of the direction's length); a record stays zero where its path
    // traced no such ray. For per-ray work counts (nodes and triangles visited), not for renders.
    float *rayTap;
    int32_t rayTapPaths;
    int32_t rayTapBounces;
};

// Parameters of prgpu_render_aov (pr::RenderAOV, src/integrators/aov.h:10-21).
struct AovParams {
    int32_t type;             // 0 albedo, 1 normal, 2 depth, 3 position (pr::AOVType)
    int32_t spp;              // jittered samples per pixel
    uint64_t seed;
    int32_t throughSpecular;  // follow perfectly specular chains (denoiser guides)
    int32_t d65Spectrum;      // SceneDesc::spectra index of the D65 illuminant (albedo)
    float whiteAdaptation[9]; // albedo: XYZ white adaptation, then ...
    float xyzToRGB[9];        // ... XYZ -> linear sRGB, both row-major (color.cpp:92-99)
};

// One render of a batch (prgpu_render_batch): its scene, optional extension, parameters and film.
struct BatchItem {
    const SceneDesc *scene;
    const SceneExt *ext;            // optional (light BVH, grid media); wavefrontPaths/blockSize unused
    RenderParams params;            // spp, firstSample, seed, maxDepth, clampLuminance of this render
    double *outXYZ;                 // host film, width * height * 3: samples ADDED in sample order
};

// Launch settings of a batch. A zero field is filled in by the autotuner (prgpu_autotune_batch),
// whose choice is cached per device and batch shape.
struct BatchConfig {
    uint32_t structSize;            // sizeof(BatchConfig)
    int32_t wavefrontPaths;         // paths in flight = queue capacity (1,024 .. 2^24)
    int32_t shadeBlock;             // threads per block of the shading kernel (64, 128, 192 or 256)
    int32_t flags;                  // bit 0: drive the loop from the host, one synchronisation per
                                    // iteration, instead of the graph (for profilers, which cannot
                                    // see inside conditional graphs); other bits 0
};

// Counters of one prgpu_render_batch call.
struct BatchStats {
    uint64_t pathSamples;           // camera samples traced over all renders
    uint64_t closestRays;
    uint64_t shadowRays;
    uint64_t waves;                 // wavefronts (each a set of chunks, at most one per render)
    uint64_t loopIterations;        // iterations of the device-side loop (2 bounces each)
    double deviceMs;                // the graph launch, CUDA events
    double hostMs;                  // scene residency, scheduling and film copies (wall clock)
    int32_t wavefrontPaths;         // the settings used
    int32_t shadeBlock;
    int32_t graphBuilt;             // 1 when this call had to (re)build the CUDA graph
    int32_t tuned;                  // 1 when this call ran the autotuner
};

// Per-call counters and device timings.
struct RenderStats {
    uint64_t pathSamples;      // camera samples traced
    uint64_t closestRays;      // closest-hit queries
    uint64_t shadowRays;       // shadow (any-hit / transmittance) queries
    uint64_t bounces;          // wavefront iterations
    uint64_t kernelLaunches;   // kernels launched by this call
    double deviceMs;           // device time of the render (CUDA events)
    double traceMs;            // device time in the closest-hit kernel
    double shadowMs;           // device time in the shadow kernel
    double shadeMs;            // device time in the shading kernel
    double filmMs;             // device time in the film kernel
};

// Settings of the path-guiding network's sampling and online training (prgpu_guide_set_options;
// defaults in brackets).
struct GuideOptions {
    float maxSelect;           // [0.5] cap of the probability c of sampling the guide (0 < x <= 0.99)
    float logKappaMax;         // [8] upper clamp of the lobes' log concentration (0 <= x <= 8)
    int32_t selectLoss;        // [0] c trained on the mixture's KL divergence (0) or on the second
                               //     moment of the one-sample estimator (1)
    int32_t trainPasses;       // [1] online training passes over each chunk's samples (1..64)
    int32_t bands;             // [12] position-encoding bands in use (0..12; the others input 0)
    float weightClamp;         // [20; 0 = off] online training weights, normalised to mean 1 per batch, clamped
};

} // namespace prgpu

// --------------------------------------------------------------------------------------------
// v4 entry points -- the exact set prender_gpu exports (src/gpu/gpu_api.h:166-173), resolved by
// name in src/integrators/gpu_path.cpp:59-61.

// Returns prgpu::kApiVersion (4). Replaces prgpu_api_version, gpu_api.h:173.
PRGPU_API int prgpu_api_version();

// Fills out[kSheenAlpha * kSheenMu] with the sheen lobe's directional albedo at the table nodes
// ([roughness 0.05..1][cos theta 0..1]), computed on the host as the reference's
// SheenBxDF::Albedo does (src/materials/bxdf.cpp:538-560): the table a host may pass in
// SceneDesc::sheenAlbedo. A scene with sheen and a null table gets this one. No device work.
PRGPU_API void prgpu_sheen_albedo_table(float *out);

// Writes up to max CUDA devices; returns the number written. Replaces prgpu_list_devices,
// gpu_api.h:166-167 (backend reads "cuda").
PRGPU_API int prgpu_list_devices(prgpu::DeviceInfo *out, int max);

// Renders params->spp samples per pixel (sample indices firstSample .. firstSample+spp-1) and
// ADDS the unnormalised per-pixel XYZ sums into outXYZ (3 floats per pixel, raster order).
// Deterministic in (seed, pixel, sample index). Replaces prgpu_render, gpu_api.h:168-172.
PRGPU_API int prgpu_render(int deviceIndex, const prgpu::SceneDesc *scene, const prgpu::RenderParams *params,
                           float *outXYZ, char *err, int errLen);

// --------------------------------------------------------------------------------------------
// Extension entry points (no counterpart in src/gpu/gpu_api.h)

// Returns prgpu::kExtVersion (5).
PRGPU_API int prgpu_ext_version();

// Like prgpu_render, but ADDS FP64 sums (each pixel's samples added one at a time in sample-index
// order, so splitting a render into batches gives bit-identical sums), accepts the optional
// SceneExt (light BVH, wavefront sizing) and reports RenderStats (either may be null).
PRGPU_API int prgpu_render_ex(int deviceIndex, const prgpu::SceneDesc *scene, const prgpu::SceneExt *ext,
                              const prgpu::RenderParams *params, double *outXYZ, prgpu::RenderStats *stats,
                              char *err, int errLen);

// Ray queries against a caller BVH over a triangle soup (the reference CPU routines are
// pr::BVH::Intersect / IntersectP, src/geometry/bvh.cpp:158-232; triangle test
// pr::Triangle::Intersect, src/geometry/shape.cpp:202-222). Triangles are 3 vertices each, indexed
// by primitive; nodes/primOrder as in SceneDesc. Closest hit (anyHit = 0) writes primOut = the
// hit primitive (-1 = miss), tOut = its distance, b1Out/b2Out = barycentrics (each may be null).
// Any hit (anyHit = 1) writes primOut = 1 (occluded) or 0. Inputs and outputs are host memory.
PRGPU_API int prgpu_trace_rays(int deviceIndex, const prgpu::BVHNode *nodes, int32_t nodeCount,
                               const int32_t *primOrder, const prgpu::Float3 *triVerts, int32_t primCount,
                               const prgpu::Ray *rays, int64_t rayCount, int32_t anyHit, int32_t *primOut,
                               float *tOut, float *b1Out, float *b2Out, char *err, int errLen);

// The same query as prgpu_trace_rays, for callers that cannot allocate device memory while they
// work (their HBM belongs to another allocator's pool, or they must not trigger the device-wide
// synchronisation of cudaMalloc / cudaFree). It allocates nothing: every device byte comes from
// one 32 MiB array the library reserves on each GPU where it is loaded. Limits: at most 131,072
// triangles and 262,143 BVH nodes per call (larger inputs return 1 with a message); any number of
// rays. Calls run one after another, on the calling thread's per-thread default stream. The
// first call on a device also does the runtime's one-time set-up (the array's address, module
// load, local-memory reserve): make it before the point from which nothing may allocate. This
// entry point has no counterpart in the reference.
PRGPU_API int prgpu_trace_rays_noalloc(int deviceIndex, const prgpu::BVHNode *nodes, int32_t nodeCount,
                                       const int32_t *primOrder, const prgpu::Float3 *triVerts, int32_t primCount,
                                       const prgpu::Ray *rays, int64_t rayCount, int32_t anyHit, int32_t *primOut,
                                       float *tOut, float *b1Out, float *b2Out, char *err, int errLen);

// Device-resident acceleration structure for repeated queries: built once from the same inputs
// as prgpu_trace_rays, queried with device pointers on a caller stream (cudaStream_t as void*).
typedef struct prgpu_accel_t *prgpu_accel;
PRGPU_API int prgpu_accel_create(int deviceIndex, const prgpu::BVHNode *nodes, int32_t nodeCount,
                                 const int32_t *primOrder, const prgpu::Float3 *triVerts, int32_t primCount,
                                 prgpu_accel *out, char *err, int errLen);
PRGPU_API int prgpu_accel_trace(prgpu_accel accel, const prgpu::Ray *deviceRays, int64_t rayCount, int32_t anyHit,
                                int32_t *devicePrimOut, float *deviceTOut, void *stream, char *err, int errLen);
// Same query with HOST rays and results: the rays are copied in and the results out inside the
// call, overlapped chunk by chunk with the traversal.
PRGPU_API int prgpu_accel_trace_host(prgpu_accel accel, const prgpu::Ray *rays, int64_t rayCount, int32_t anyHit,
                                     int32_t *primOut, float *tOut, char *err, int errLen);
// Returns and clears the handle's status word: bit 0 = a traversal stack overflowed (the BVH is
// deeper than 64 levels along some ray); -1 on a bad handle.
PRGPU_API int prgpu_accel_status(prgpu_accel accel);
// Bytes of the converted node and triangle arrays on the device (for roofline accounting).
PRGPU_API int64_t prgpu_accel_bytes(prgpu_accel accel);
PRGPU_API void prgpu_accel_destroy(prgpu_accel accel);

// Renders count (1..256) scenes of any size, sample count and path length together: their paths
// share one set of per-bounce queues in one wavefront, and the whole batch runs as ONE launch of a
// CUDA graph whose device-side loop (a conditional while node) raygens, traces, shades and films
// wave after wave with no host round trip. Each film gets exactly the bits prgpu_render_ex would
// add for that item alone. config may be null (all settings autotuned). No counterpart in the
// reference, whose host renders one scene per call (src/integrators/gpu_path.cpp:458-509).
// Auxiliary buffer of a scene at its film resolution (pr::RenderAOV, src/integrators/aov.cpp:147-196):
// albedo (linear sRGB directional albedo of the first visible surface, coverage-weighted), world
// shading normal (normalised sum), depth (nearest along the camera ray, 1e10 where nothing is hit)
// or position (mean over hits); throughSpecular follows mirrors and glass to the first
// non-specular surface (or into a scattering medium: its single-scattering albedo). outRGB:
// width * height * 3 floats, overwritten. Returns 0, or 1 with err set.
PRGPU_API int prgpu_render_aov(int deviceIndex, const prgpu::SceneDesc *scene, const prgpu::SceneExt *ext,
                               const prgpu::AovParams *params, float *outRGB, char *err, int errLen);

PRGPU_API int prgpu_render_batch(int deviceIndex, int32_t count, const prgpu::BatchItem *items,
                                 const prgpu::BatchConfig *config, prgpu::BatchStats *stats, char *err, int errLen);

// Times short trial renders of the batch (about 2^24 path samples, films untouched) for every
// candidate queue capacity and shading block size, caches the fastest for this device and batch
// shape, and writes it to out.
PRGPU_API int prgpu_autotune_batch(int deviceIndex, int32_t count, const prgpu::BatchItem *items,
                                   prgpu::BatchConfig *out, char *err, int errLen);

// Path-guiding network (no counterpart in the reference renderer, whose PathIntegrator samples
// the BSDF only, src/integrators/path.cpp:215-224). 128 inputs (guide features: position in the
// scene bounds with 12 sin/cos bands, normal, outgoing direction, a constant 1), 4 hidden ReLU
// layers of 64 (unit 63 held at 1), 48 outputs (8 von Mises-Fisher lobes + a selection
// probability); FP16 weights on the tensor cores, FP32 master weights and Adam state per device.
// Weights are prgpu::kGuideParams floats, layer by layer, each layer [out x in] row-major.
PRGPU_API int prgpu_guide_set_weights(int deviceIndex, const float *weights, char *err, int errLen);
PRGPU_API int prgpu_guide_get_weights(int deviceIndex, float *weights, char *err, int errLen);
// Network outputs (n x 48 floats) for n feature rows (n x 128 floats, rounded to FP16 on the device).
PRGPU_API int prgpu_guide_infer(int deviceIndex, int64_t n, const float *features, float *out, char *err, int errLen);
// One training pass: samples are n x 8 floats (wi[3], BSDF pdf of wi, weight w, shading normal[3]);
// writes the summed loss -sum w (log q_n(wi) + log(c q_n(wi) + (1 - c) pdf)) (q_n: the mixture
// folded onto the normal's hemisphere holding wi) and its gradient w.r.t. the weights
// (kGuideParams floats; the selection term's gradient taken at fixed q_n).
PRGPU_API int prgpu_guide_gradient(int deviceIndex, int64_t n, const float *features, const float *samples,
                                   float *lossSum, float *grad, char *err, int errLen);
// Learning rate of online training (default 1e-3), per device.
PRGPU_API int prgpu_guide_set_learning_rate(int deviceIndex, float learningRate, char *err, int errLen);
// Training state: out4 = {summed loss of the last training pass (with the batch's weights
// normalised to mean 1 in online training), rows of the last online batch, their weight sum,
// Adam steps taken}.
PRGPU_API int prgpu_guide_stats(int deviceIndex, float *out4, char *err, int errLen);
// Adam step (beta 0.9 / 0.999, eps 1e-8) on the last gradient times gradScale.
PRGPU_API int prgpu_guide_adam_step(int deviceIndex, float gradScale, float learningRate, char *err, int errLen);
// Sampling and training settings of the guide on a device (null: the defaults); out-of-range
// values return 1 with a message. They apply to later renders, gradients and training steps.
PRGPU_API int prgpu_guide_set_options(int deviceIndex, const prgpu::GuideOptions *opts, char *err, int errLen);
PRGPU_API int prgpu_guide_get_options(int deviceIndex, prgpu::GuideOptions *out, char *err, int errLen);

// Number of kernel launches this library has issued since load (for launch accounting).
PRGPU_API uint64_t prgpu_launch_count();

// Verification entry points: the path tracer's own device functions evaluated on caller inputs
// (host arrays), for comparison with the reference implementations on identical inputs.
// BxDF (kind 0 diffuse, 1 conductor, 2 dielectric, 3 thin dielectric; pr::DiffuseBxDF,
// ConductorBxDF, DielectricBxDF, ThinDielectricBxDF, src/materials/bxdf.cpp:85-256):
//   params 16 floats: R[4], eta[4], k[4], etaD, alphaX, alphaY, mode (0 radiance, 1 importance);
//   in 9 floats per item: wo[3], wi[3], uc, u0, u1;
//   out 16 floats per item: f[4], pdf, sampled (0/1), sample f[4], pdf, wi[3], flags, eta.
PRGPU_API int prgpu_eval_bxdf(int deviceIndex, int kind, const float *params, int64_t n, const float *in, float *out,
                              char *err, int errLen);
// Coated and sheen BSDFs on identical local-frame inputs (pr::LayeredBxDF over a diffuse or
// conductor base, src/materials/bxdf.cpp:260-518, and pr::SheenBxDF over it or over a single lobe,
// bxdf.cpp:520-631). params (36 floats): layered, base kind (0 diffuse, 1 conductor, 2 dielectric),
// R[4], eta[4], k[4], etaD, alphaX, alphaY, coat eta, coat alpha, thickness, g, albedo[4],
// maxDepth, nSamples, sheen weight, sheen roughness, sheen colour[4], 2 unused; sheenTable: the
// [16 roughness][32 cos theta] sheen albedo table (needed when the sheen weight is > 0). in / out
// as prgpu_eval_bxdf, with out[15] = 1 when the sampled pdf is only proportional.
PRGPU_API int prgpu_eval_full_bsdf(int deviceIndex, const float *params, const float *sheenTable, int64_t n,
                                   const float *in, float *out, char *err, int errLen);
// Henyey-Greenstein (src/materials/bxdf.cpp:64-80): in 7 floats (cosTheta, g, wo[3], u0, u1);
// out 5 floats (phase value, sampled wi[3], its pdf).
PRGPU_API int prgpu_eval_phase(int deviceIndex, int64_t n, const float *in, float *out, char *err, int errLen);
// Homogeneous medium (HomogeneousMedium::Transmittance / SampleDistanceHero,
// src/media/medium.cpp:15-103): in 10 floats (sigma_a[4], sigma_s[4], tMax, u); out 14 floats
// (Tr(tMax)[4], scattered, t, weight[4], pdfRatio[4]).
PRGPU_API int prgpu_eval_homogeneous(int deviceIndex, int64_t n, const float *in, float *out, char *err, int errLen);
// Light-BVH next-event selection (pr::BVHLightSampler::Sample / PMF, src/lights/light_bvh.cpp:179-234)
// over caller nodes: in 7 floats (p[3], n[3], u); out 2 floats (chosen light or -1, its pmf);
// pmfOut (optional) n x lightCount: the pmf of every light at that point. bvhProb scales the
// BVH branch (1 when there is no infinite light).
PRGPU_API int prgpu_eval_light_bvh(int deviceIndex, const prgpu::LightBVHNode *nodes, int32_t nodeCount,
                                   int32_t lightCount, float bvhProb, int64_t n, const float *in, float *out,
                                   float *pmfOut, char *err, int errLen);
