// prhost_api.h -- C ABI of libprender_host.so, the C++ host side that prepares scenes for the
// CUDA module: it builds the acceleration structures a SceneDesc carries.
//
// In PRender the host builds its BVH in pr::BVH::Build (src/geometry/bvh.cpp:8-135) and hands the
// flattened nodes to the GPU module (src/integrators/gpu_path.cpp:378-390); its light BVH is
// pr::BVHLightSampler (src/lights/light_bvh.cpp:103-177). These entry points produce the same
// node formats (prgpu::BVHNode, prgpu::LightBVHNode) from plain arrays, so a caller without
// PRender's scene classes can drive libprender_gpu.so.
#pragma once

#include <cstdint>

#include "prgpu_api.h"

#if defined(_WIN32)
#define PRHOST_API extern "C" __declspec(dllexport)
#else
#define PRHOST_API extern "C" __attribute__((visibility("default")))
#endif

// Binned-SAH BVH over primitive bounds (boxMin/boxMax: 3 floats per primitive). Writes at most
// 2 * primCount - 1 nodes in depth-first order (first child follows its parent, offset = second
// child; leaves hold primOrder[offset .. offset + nPrims)) and the leaf-slot permutation.
// maxLeaf bounds primitives per leaf (1..8); threads = 0 uses all hardware threads.
// Returns the node count, or -1 on bad arguments. Replaces pr::BVH::Build (bvh.cpp:8-135).
PRHOST_API int64_t prhost_build_bvh(const float *boxMin, const float *boxMax, int64_t primCount, int32_t maxLeaf,
                                    int32_t threads, prgpu::BVHNode *nodesOut, int32_t *primOrderOut);

// Triangle-soup convenience: bounds from 3 vertices per primitive.
PRHOST_API int64_t prhost_build_bvh_triangles(const prgpu::Float3 *verts, int64_t primCount, int32_t maxLeaf,
                                              int32_t threads, prgpu::BVHNode *nodesOut, int32_t *primOrderOut);

// Light BVH over bounded lights (Conty & Kulla importance, 12-bucket SAOH on 3 axes, as
// src/lights/light_bvh.cpp:90-177). Per light: bounds (6 floats), emission cone axis w (3),
// phi, cosThetaO, cosThetaE, twoSided (as float 0/1): 13 floats. Writes 2 * n - 1 nodes; returns
// the node count or -1.
PRHOST_API int32_t prhost_build_light_bvh(const float *lightBounds13, int32_t lightCount,
                                          prgpu::LightBVHNode *nodesOut);

namespace prhost {

// Header of a progressive-render checkpoint (the fields src/integrators/integrator.cpp:18-28
// writes after the "PRCKPT02" magic). A resume is refused unless every field matches.
struct CheckpointHeader {
    uint32_t integrator;   // pr::IntegratorType (0 path, 1 BDPT, 2 MMLT, 3 PSSMLT) | 0x100 for a GPU render
    int32_t maxDepth;      // the integrator's max depth (0 = unlimited)
    int32_t width, height; // film size
    int32_t chains;        // pr::IntegratorSettings::chains (written for every integrator)
    uint64_t fingerprint;  // scene fingerprint (pr::Scene::Fingerprint, scene.cpp:61-70)
    uint64_t seed;         // render seed
};

} // namespace prhost

// Writes a checkpoint in the reference's PRCKPT02 layout (integrator.cpp:30-60, film.cpp:61-73):
// magic, header, filmCount (= width * height * 3) FP64 XYZ accumulators, then bodySize bytes of
// integrator state (the GPU path tracer stores its samples per pixel as one int32). Written to
// "<path>.tmp" and renamed over path. Returns 0, or 1 with err set. Replaces pr::WriteCheckpoint.
PRHOST_API int prhost_checkpoint_write(const char *path, const prhost::CheckpointHeader *header, const double *film,
                                       uint64_t filmCount, const void *body, uint64_t bodySize, char *err,
                                       int errLen);

// Reads a checkpoint written for exactly *expected (integrator.cpp:62-90, film.cpp:75-84): the
// film into film[filmCount], the body into body[bodyCapacity] (its size in *bodySize). Returns 0;
// 1 cannot open or bad arguments; 2 not a checkpoint; 3 made for another scene / integrator /
// device / resolution / seed / depth; 4 truncated or corrupt -- with the reference's messages in
// err. Replaces pr::ReadCheckpoint.
PRHOST_API int prhost_checkpoint_read(const char *path, const prhost::CheckpointHeader *expected, double *film,
                                      uint64_t filmCount, void *body, uint64_t bodyCapacity, uint64_t *bodySize,
                                      char *err, int errLen);

// Preetham daylight (A. J. Preetham, P. Shirley, B. Smits, SIGGRAPH 1999) as PRender builds it for
// a "sun_sky" light: an equirect (+y up) map of width x height linear-sRGB texels (rgb: 3 floats
// each, row 0 at the zenith) for the sun direction sunDir (normalised here), turbidity T (clamped
// to [1.7, 10]) and a Lambertian ground of groundAlbedo below the horizon. Returns 0, or 1 on bad
// arguments. Replaces pr::MakePreethamSky (src/lights/sky.cpp:146-205).
PRHOST_API int prhost_preetham_sky(const float *sunDir, float turbidity, float groundAlbedo, int32_t width,
                                   int32_t height, float *rgb);
// The sun's spectral radiance (a 5778 K blackbody at the solar disk's luminance, scaled for an
// enlarged disk, through the Rayleigh and aerosol optical depth of the air mass) at n wavelengths
// (nm). Returns 0, or 1 on bad arguments. Replaces pr::MakeSunRadiance (src/lights/sky.cpp:207-233).
PRHOST_API int prhost_sun_radiance(const float *sunDir, float turbidity, float angularRadiusDeg, int64_t n,
                                   const float *lambdaNm, float *out);
// Unbounded RGB -> environment-map texel (prgpu::EnvMapDesc::texels): per colour, out4 = (c0, c1,
// c2, scale) with the spectrum scale * S(c0 l^2 + c1 l + c2), l in nm, S(x) = 1/2 + x / (2
// sqrt(1 + x^2)), scale = 2 max(r, g, b) (0 for a colour without a positive component), the
// coefficients fitted (Gauss-Newton in CIELAB, D65 white) so that the reflectance S of rgb / scale
// under illuminant95 (95 samples at 360..830 nm by 5, scaled to unit luminance) has the colour's
// sRGB XYZ. threads = 0
// uses all hardware threads. Returns 0, or 1 on bad arguments. The reference interpolates its
// precomputed table of the same fits under D65 instead (RGBToSpectrumTable, src/core/rgb2spec.cpp).
PRHOST_API int prhost_rgb_to_sigmoid(int64_t n, const float *rgb, const float *illuminant95, int32_t threads,
                                     float *out4);
